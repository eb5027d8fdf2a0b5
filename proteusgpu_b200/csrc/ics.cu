// Initial conditions generated on the device (extension: the reference reads
// them from HDF5 files written by its create*.py scripts, src/io/input.cpp:121-309).
//
// The workloads' generators in proteusgpu_b200/ics.py and these kernels produce
// the same points and fields bit for bit: every random number is a pure
// function of (seed, stream, index) -- the SplitMix64 output function (Steele,
// Lea, Flood, OOPSLA 2014) of key + (index + 1) * 0x9E3779B97F4A7C15 -- and the
// transcendental functions the generators need are evaluated by the same
// sequences of IEEE double operations on both sides (this file is compiled
// with -fmad=false): ln by exponent split and the atanh series, exp by
// reduction with ln 2 and a Taylor series, sin/cos by quadrant reduction and
// Taylor series, normals by Marsaglia's polar method.  The Sedov blast deposit
// selects the 32 points nearest the box centre (ties by index) with a two-pass
// block selection and weights them with exp(-r^2 / (2 sigma^2)).
#include <math_constants.h>
#include <stdint.h>

#include <algorithm>

#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;
constexpr int S_JITTER = 1, S_POS = 2, S_CENTRE = 3, S_SIGMA = 4, S_WHICH = 5, S_GAUSS = 6, S_NOISE = 7;
constexpr double LN2 = 0.6931471805599453, INV_LN2 = 1.4426950408889634;
constexpr double HALF_PI = 1.5707963267948966, INV_HALF_PI = 0.6366197723675814, FOUR_PI = 12.566370614359172;
constexpr double SQRT_HALF = 0.7071067811865476, TWO_M53 = 1.1102230246251565e-16;
constexpr int DEP_N = 32;          // points the blast is spread over
constexpr double DEP_SIGMA = 0.01;  // width of its Gaussian weights
constexpr int SEL_T = 256;         // threads of a selection block
constexpr int SEL_BUF = 512;       // keys a selection block sorts at once

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t stream_key(uint64_t seed, int stream) { return mix64(seed * GOLDEN + (uint64_t)stream); }

__device__ __forceinline__ uint64_t word(uint64_t key, uint64_t i) { return mix64(key + (i + 1ull) * GOLDEN); }
__device__ __forceinline__ double unif(uint64_t key, uint64_t i) { return (double)(word(key, i) >> 11) * TWO_M53; }

__device__ double log_d(double x) {
    int e;
    double m = frexp(x, &e);
    if (m < SQRT_HALF) {
        m = m * 2.0;
        e = e - 1;
    }
    const double t = (m - 1.0) / (m + 1.0);
    const double t2 = t * t;
    double s = 0.047619047619047616;
    s = s * t2 + 0.05263157894736842;
    s = s * t2 + 0.058823529411764705;
    s = s * t2 + 0.06666666666666667;
    s = s * t2 + 0.07692307692307693;
    s = s * t2 + 0.09090909090909091;
    s = s * t2 + 0.1111111111111111;
    s = s * t2 + 0.14285714285714285;
    s = s * t2 + 0.2;
    s = s * t2 + 0.3333333333333333;
    s = s * t2 + 1.0;
    return (double)e * LN2 + 2.0 * t * s;
}

__device__ double exp_d(double x) {
    const double k = rint(x * INV_LN2);
    const double r = x - k * LN2;
    const double c[14] = {1.0, 1.0, 0.5, 0.16666666666666666, 0.041666666666666664, 0.008333333333333333,
                          0.001388888888888889, 0.0001984126984126984, 2.48015873015873e-05,
                          2.7557319223985893e-06, 2.755731922398589e-07, 2.505210838544172e-08,
                          2.08767569878681e-09, 1.6059043836821613e-10};
    double s = c[13];
#pragma unroll
    for (int j = 12; j >= 1; j--) s = s * r + c[j];
    s = s * r + 1.0;
    return ldexp(s, (int)k);
}

__device__ void sincos_red(double r, double& s, double& c) {
    const double sc[9] = {1.0, -0.16666666666666666, 0.008333333333333333, -0.0001984126984126984,
                          2.7557319223985893e-06, -2.505210838544172e-08, 1.6059043836821613e-10,
                          -7.647163731819816e-13, 2.8114572543455206e-15};
    const double cc[10] = {1.0, -0.5, 0.041666666666666664, -0.001388888888888889, 2.48015873015873e-05,
                           -2.755731922398589e-07, 2.08767569878681e-09, -1.1470745597729725e-11,
                           4.779477332387385e-14, -1.5619206968586225e-16};
    const double r2 = r * r;
    s = sc[8];
#pragma unroll
    for (int j = 7; j >= 0; j--) s = s * r2 + sc[j];
    s = s * r;
    c = cc[9];
#pragma unroll
    for (int j = 8; j >= 0; j--) c = c * r2 + cc[j];
}

__device__ double sin_d(double x) {
    const double k = rint(x * INV_HALF_PI);
    const double r = x - k * HALF_PI;
    double s, c;
    sincos_red(r, s, c);
    const long long q = (long long)k & 3;
    return q == 0 ? s : (q == 1 ? c : (q == 2 ? -s : -c));
}

__device__ double normal_d(uint64_t key, uint64_t i) {
    for (int j = 0; j < 64; j++) {
        const uint64_t c = i * 128ull + 2ull * (uint64_t)j;
        const double u = 2.0 * unif(key, c) - 1.0;
        const double v = 2.0 * unif(key, c + 1ull) - 1.0;
        const double s = u * u + v * v;
        if (s < 1.0 && s > 0.0) return u * sqrt(-2.0 * log_d(s) / s);
    }
    return 0.0;
}

__device__ __forceinline__ double wrap01(double p) {
    double r = fmod(p, 1.0);
    if (r < 0.0) r = r + 1.0;
    return r >= 1.0 ? 0.0 : r;
}

struct IcArgs {
    int kind, dim;
    int64_t n;
    int n_side;
    double h;  // 1 / n_side
    double jitter, gamma, split_cos, split_sin, p0, rho_ratio;
    uint64_t k_jit, k_pos, k_which, k_gauss, k_noise, k_centre, k_sigma;
    int n_clumps;
    int64_t n_cl;  // clumped points (the first n_cl)
};

// Clump centres and widths (ics.clump_params): 64 entries.
__global__ void k_ic_clumps(IcArgs A, double* __restrict__ cen, double* __restrict__ sig) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.n_clumps) return;
    for (int a = 0; a < 3; a++) cen[3 * c + a] = unif(A.k_centre, 3ull * (uint64_t)c + (uint64_t)a);
    const double lo = log_d(0.005), hi = log_d(0.05);
    sig[c] = exp_d(lo + (hi - lo) * unif(A.k_sigma, (uint64_t)c));
}

// Positions and primitives of point i; pos is n x dim.
__global__ void k_ic_points(IcArgs A, const double* __restrict__ cen, const double* __restrict__ sig,
                            double* __restrict__ pos, double* __restrict__ rho, double* __restrict__ vel,
                            double* __restrict__ en) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const int D = A.dim;
    double p[3] = {0.0, 0.0, 0.0};
    if (A.kind == PGPU_IC_SOD || A.kind == PGPU_IC_KH) {
        int64_t rest = i;
        for (int a = 0; a < D; a++) {
            const int64_t ia = rest % A.n_side;
            rest = rest / A.n_side;
            const double base = ((double)ia + 0.5) * A.h;
            const double j = (2.0 * unif(A.k_jit, (uint64_t)(D * i + a)) - 1.0) * A.jitter;
            p[a] = fmin(fmax(base + j * A.h, 0.0), 0.9999999999999999);
        }
    } else if (A.kind == PGPU_IC_CLUSTERED && i < A.n_cl) {
        const int w = (int)(((word(A.k_which, (uint64_t)i) >> 32) * (uint64_t)A.n_clumps) >> 32);
        for (int a = 0; a < 3; a++) {
            const double g = normal_d(A.k_gauss, (uint64_t)(3 * i + a));
            p[a] = wrap01(cen[3 * w + a] + g * sig[w]);
        }
    } else {
        for (int a = 0; a < D; a++) p[a] = unif(A.k_pos, (uint64_t)(D * i + a));
    }
    for (int a = 0; a < D; a++) pos[D * i + a] = p[a];
    double r, vx = 0.0, vy = 0.0, E;
    if (A.kind == PGPU_IC_SOD) {
        const bool left = ((p[0] - 0.5) * A.split_cos + (p[1] - 0.5) * A.split_sin) < 0.0;
        r = left ? 1.0 : 0.125;
        E = (left ? 1.0 : 0.1) / (A.gamma - 1.0);
    } else if (A.kind == PGPU_IC_KH) {
        const bool band = fabs(p[1] - 0.5) < 0.25;
        r = band ? A.rho_ratio : 1.0;
        vx = band ? 0.5 : -0.5;
        vy = 0.01 * sin_d(FOUR_PI * p[0]) + 1e-3 * normal_d(A.k_noise, (uint64_t)i);
        E = 2.5 / (A.gamma - 1.0) + (0.5 * r) * (vx * vx + vy * vy);
    } else {
        r = 1.0;
        E = A.p0 / (A.gamma - 1.0);
    }
    rho[i] = r;
    en[i] = E;
    vel[D * i] = vx;
    vel[D * i + 1] = vy;
    if (D == 3) vel[D * i + 2] = 0.0;
}

// ---- the blast's points: the DEP_N smallest keys (d^2 to the centre, index) ----
struct Key {
    double d;
    uint32_t i;
};
__device__ __forceinline__ bool key_lt(const Key& a, const Key& b) { return a.d < b.d || (a.d == b.d && a.i < b.i); }

__device__ __forceinline__ Key point_key(const double* pos, int D, int64_t i) {
    double d2 = 0.0;
    for (int a = 0; a < D; a++) {
        const double d = pos[D * i + a] - 0.5;
        d2 = d2 + d * d;
    }
    return Key{d2, (uint32_t)i};
}

// Ascending bitonic sort of SEL_BUF keys in shared memory by SEL_T threads.
__device__ void sort_buf(Key* buf) {
    for (int k = 2; k <= SEL_BUF; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < SEL_BUF; t += SEL_T) {
                const int o = t ^ j;
                if (o > t) {
                    const bool up = (t & k) == 0;
                    const Key a = buf[t], b = buf[o];
                    if (up ? key_lt(b, a) : key_lt(a, b)) {
                        buf[t] = b;
                        buf[o] = a;
                    }
                }
            }
            __syncthreads();
        }
}

// Each block keeps the DEP_N smallest keys of its range [b * chunk, +chunk) of
// either points (pos != NULL) or keys (in): candidates below the running DEP_N-th
// key are appended to a buffer that is sorted, down to DEP_N, when it could overflow.
__global__ void __launch_bounds__(SEL_T) k_select(const double* __restrict__ pos, int D, const Key* __restrict__ in,
                                                 int64_t n, int64_t chunk, Key* __restrict__ out) {
    __shared__ Key buf[SEL_BUF];
    __shared__ int cnt;
    const int64_t lo = (int64_t)blockIdx.x * chunk, hi = min(n, lo + chunk);
    for (int t = threadIdx.x; t < SEL_BUF; t += SEL_T) buf[t] = Key{CUDART_INF, 0xFFFFFFFFu};
    if (threadIdx.x == 0) cnt = DEP_N;
    __syncthreads();
    Key thr{CUDART_INF, 0xFFFFFFFFu};
    for (int64_t base = lo; base < hi; base += SEL_T) {
        const int64_t i = base + threadIdx.x;
        if (i < hi) {
            const Key k = pos ? point_key(pos, D, i) : in[i];
            if (key_lt(k, thr)) buf[atomicAdd(&cnt, 1)] = k;
        }
        __syncthreads();
        if (cnt > SEL_BUF - SEL_T || base + SEL_T >= hi) {
            sort_buf(buf);
            for (int t = DEP_N + threadIdx.x; t < SEL_BUF; t += SEL_T) buf[t] = Key{CUDART_INF, 0xFFFFFFFFu};
            if (threadIdx.x == 0) cnt = DEP_N;
            __syncthreads();
            thr = buf[DEP_N - 1];
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < DEP_N; t += SEL_T) out[(int64_t)blockIdx.x * DEP_N + t] = buf[t];
}

// Weights of the DEP_N nearest points (nearest first), their sum in that order, and
// the deposit e_total * w / sum at their indices (deposit zeroed before).
__global__ void k_deposit(const Key* __restrict__ best, double e_blast, double* __restrict__ dep) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double w[DEP_N];
    double tot = 0.0;
    for (int j = 0; j < DEP_N; j++) {
        w[j] = exp_d(-best[j].d / (2.0 * DEP_SIGMA * DEP_SIGMA));
        tot = tot + w[j];
    }
    for (int j = 0; j < DEP_N; j++) dep[best[j].i] = e_blast * (w[j] / tot);
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Generates spec's initial condition into device arrays pos (n x dim), rho, vel
// (n x dim), en and, for the blast kinds, dep (zeroed, then the deposit).
cudaError_t ic_generate(pgpu_ctx* c, const pgpu_ic_spec* s, int64_t n, double* pos, double* rho, double* vel,
                        double* en, double* dep) {
    IcArgs A{};
    A.kind = s->kind;
    A.dim = s->dim;
    A.n = n;
    A.n_side = s->n_side;
    A.h = s->n_side > 0 ? 1.0 / (double)s->n_side : 0.0;
    A.jitter = s->jitter;
    A.gamma = s->gamma;
    A.split_cos = s->split_cos;
    A.split_sin = s->split_sin;
    A.p0 = s->p0;
    A.rho_ratio = s->rho_ratio;
    A.k_jit = stream_key(s->seed, S_JITTER);
    A.k_pos = stream_key(s->seed, S_POS);
    A.k_which = stream_key(s->seed, S_WHICH);
    A.k_gauss = stream_key(s->seed, S_GAUSS);
    A.k_noise = stream_key(s->seed, S_NOISE);
    A.k_centre = stream_key(s->seed, S_CENTRE);
    A.k_sigma = stream_key(s->seed, S_SIGMA);
    A.n_clumps = s->n_clumps;
    A.n_cl = s->kind == PGPU_IC_CLUSTERED ? (int64_t)llrint(s->frac_clumped * (double)n) : 0;
    cudaError_t e = cudaSuccess;
    DevBuf tmp;
    const int nsel = (int)std::min<int64_t>(1024, std::max<int64_t>(1, (n + 16383) / 16384));
    const size_t clump_bytes = A.n_clumps > 0 ? (size_t)A.n_clumps * 4 * sizeof(double) : 16;
    if ((e = ensure_bytes(tmp, clump_bytes + (size_t)(nsel + 1) * DEP_N * sizeof(Key) + 256))) return e;
    double* cen = (double*)tmp.p;
    double* sig = cen + 3 * (A.n_clumps > 0 ? A.n_clumps : 1);
    Key* part = (Key*)((char*)tmp.p + ((clump_bytes + 15) / 16) * 16);
    Key* best = part + (size_t)nsel * DEP_N;
    int launches = 0;
    if (A.kind == PGPU_IC_CLUSTERED) {
        k_ic_clumps<<<1, 64, 0, c->stream>>>(A, cen, sig);
        launches++;
    }
    k_ic_points<<<nblk(n, 256), 256, 0, c->stream>>>(A, cen, sig, pos, rho, vel, en);
    launches++;
    if (dep && (A.kind == PGPU_IC_SEDOV || A.kind == PGPU_IC_CLUSTERED)) {
        if ((e = cudaMemsetAsync(dep, 0, (size_t)n * sizeof(double), c->stream))) goto done;
        if (n >= DEP_N) {
            const int64_t chunk = (n + nsel - 1) / nsel;
            k_select<<<nsel, SEL_T, 0, c->stream>>>(pos, A.dim, nullptr, n, chunk, part);
            k_select<<<1, SEL_T, 0, c->stream>>>(nullptr, A.dim, part, (int64_t)nsel * DEP_N, (int64_t)nsel * DEP_N,
                                                 best);
            k_deposit<<<1, 32, 0, c->stream>>>(best, s->e_blast, dep);
            launches += 3;
        }
    }
    count_launches(launches);
    e = cudaGetLastError();
    if (!e) e = cudaStreamSynchronize(c->stream);
done:
    if (tmp.p) cudaFree(tmp.p);
    return e;
}

}  // namespace pgpu
