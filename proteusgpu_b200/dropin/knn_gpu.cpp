// Drop-in replacement for the reference's src/knn/knn.cpp.
//
// Keeps every entry point knn.h declares (src/knn/knn.h:33-77) with the same
// signature and the same knn_problem layout (knn.h:19-31), and computes on the
// GPU through the C ABI (include/proteus_gpu.h).  knn::init sorts the points
// into the device's Morton-ordered grid and solves the K nearest neighbours in
// one call; knn::solve has nothing left to do.  As in the reference, the
// returned lists, points and permutation are all in the grid-sorted index space
// (d_knearests[s * _K_ + j] is a sorted index), ascending by squared distance
// (ties by input index); the sorted order itself is the device's grid order.
//
// Build: compile in place of src/knn/knn.cpp with -I<this repo>/include and
// -I<this repo>/proteusgpu_b200/dropin, link -lproteus_gpu.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "knn.h"
#include "pgpu_dropin.h"

namespace knn {

knn_problem* init(POINT_TYPE* pts, int len_pts) {
    knn_problem* kp = (knn_problem*)calloc(1, sizeof(knn_problem));
    kp->len_pts = len_pts;
    pgpu_ctx* c = pgpu_dropin::context();
    pgpu_dropin::invalidate_mesh();  // pgpu_knn replaces the device point set
    const size_t n = (size_t)(len_pts > 0 ? len_pts : 0);
    std::vector<uint32_t> lists(n * _K_ + 1);
    int rc = pgpu_knn(c, (const double*)pts, len_pts, lists.data());
    if (rc) pgpu_dropin::die("knn::init", rc);
    kp->d_stored_points = (POINT_TYPE*)malloc((n + 1) * sizeof(POINT_TYPE));
    kp->d_permutation = (unsigned int*)malloc((n + 1) * sizeof(unsigned int));
    int n_grid = 0;
    rc = pgpu_knn_sorted(c, (double*)kp->d_stored_points, kp->d_permutation, &n_grid);
    if (rc) pgpu_dropin::die("knn::init", rc);
    kp->N_grid = n_grid;
    kp->N_cell_offsets = 0;
    std::vector<unsigned int> to_sorted(n + 1);
    for (size_t s = 0; s < n; s++) to_sorted[kp->d_permutation[s]] = (unsigned int)s;
    kp->d_knearests = (unsigned int*)malloc((n * _K_ + 1) * sizeof(unsigned int));
    for (size_t s = 0; s < n; s++) {
        const uint32_t* row = &lists[(size_t)kp->d_permutation[s] * _K_];
        for (int j = 0; j < _K_; j++)
            kp->d_knearests[s * _K_ + j] = row[j] == UINT32_MAX ? UINT_MAX : to_sorted[row[j]];
    }
    return kp;
}

void sort_points_into_grid(knn_problem* kp, POINT_TYPE* d_points, int len_pts) {
    // The device sorts and solves in one pass: run it for the given points and
    // move the results into kp.
    knn_problem* fresh = init(d_points, len_pts);
    free(kp->d_permutation);
    free(kp->d_stored_points);
    free(kp->d_knearests);
    kp->len_pts = fresh->len_pts;
    kp->N_grid = fresh->N_grid;
    kp->d_permutation = fresh->d_permutation;
    kp->d_stored_points = fresh->d_stored_points;
    kp->d_knearests = fresh->d_knearests;
    free(fresh);
}

int cellFromPoint(int N_grid, POINT_TYPE point) {
    auto clampi = [N_grid](double x) {
        int i = (int)std::floor(x * (double)N_grid);
        return i < 0 ? 0 : (i > N_grid - 1 ? N_grid - 1 : i);
    };
#ifdef dim_2D
    return clampi(point.x) + clampi(point.y) * N_grid;
#else
    return clampi(point.x) + clampi(point.y) * N_grid + clampi(point.z) * N_grid * N_grid;
#endif
}

void solve(knn_problem* kp) { (void)kp; }

// Max-heap on vals (keys move along): restores the heap below `node`.
void heapify(unsigned int* keys, double* vals, int node, int size) {
    for (;;) {
        int big = node, l = 2 * node + 1, r = l + 1;
        if (l < size && vals[l] > vals[big]) big = l;
        if (r < size && vals[r] > vals[big]) big = r;
        if (big == node) return;
        double tv = vals[node];
        vals[node] = vals[big];
        vals[big] = tv;
        unsigned int tk = keys[node];
        keys[node] = keys[big];
        keys[big] = tk;
        node = big;
    }
}

// In-place ascending sort of a max-heap.
void heapsort(unsigned int* keys, double* vals, int size) {
    for (int end = size - 1; end > 0; end--) {
        double tv = vals[0];
        vals[0] = vals[end];
        vals[end] = tv;
        unsigned int tk = keys[0];
        keys[0] = keys[end];
        keys[end] = tk;
        heapify(keys, vals, 0, end);
    }
}

void knn_free(knn_problem** kp) {
    if (!kp || !*kp) return;
    free((*kp)->d_cell_offsets);
    free((*kp)->d_cell_offset_dists);
    free((*kp)->d_permutation);
    free((*kp)->d_counters);
    free((*kp)->d_ptrs);
    free((*kp)->d_globcounter);
    free((*kp)->d_stored_points);
    free((*kp)->d_knearests);
    free(*kp);
    *kp = NULL;
}

POINT_TYPE* get_points(knn_problem* kp) {
    POINT_TYPE* out = (POINT_TYPE*)malloc((kp->len_pts + 1) * sizeof(POINT_TYPE));
    std::copy(kp->d_stored_points, kp->d_stored_points + kp->len_pts, out);
    return out;
}

unsigned int* get_knearest(knn_problem* kp) {
    const size_t m = (size_t)kp->len_pts * _K_;
    unsigned int* out = (unsigned int*)malloc((m + 1) * sizeof(unsigned int));
    std::copy(kp->d_knearests, kp->d_knearests + m, out);
    return out;
}

unsigned int* get_permutation(knn_problem* kp) {
    unsigned int* out = (unsigned int*)malloc((kp->len_pts + 1) * sizeof(unsigned int));
    std::copy(kp->d_permutation, kp->d_permutation + kp->len_pts, out);
    return out;
}

// Brute-force check of the lists (the contract of knn::verify, knn.cpp:350-422):
// the j-th listed neighbour's squared distance must equal the j-th smallest
// within tol * (1 + d).
bool verify(knn_problem* kp, double tol, int max_report) {
    if (!kp || !kp->d_stored_points || !kp->d_knearests) {
        std::cerr << "KNN VERIFY: missing data." << std::endl;
        return false;
    }
    const int n = kp->len_pts;
    int bad = 0;
    std::vector<double> d(n > 0 ? n : 1);
    for (int i = 0; i < n; i++) {
        int m = 0;
        for (int j = 0; j < n; j++)
            if (j != i) d[m++] = dist2_point(kp->d_stored_points[i], kp->d_stored_points[j]);
        const int kk = _K_ < m ? _K_ : m;
        std::partial_sort(d.begin(), d.begin() + kk, d.begin() + m);
        bool ok = true;
        for (int j = 0; j < _K_ && ok; j++) {
            unsigned int id = kp->d_knearests[(size_t)i * _K_ + j];
            if (j >= kk) {
                ok = id == UINT_MAX;
                continue;
            }
            if (id == UINT_MAX) {
                ok = false;
                continue;
            }
            double got = dist2_point(kp->d_stored_points[i], kp->d_stored_points[id]);
            ok = std::fabs(got - d[j]) <= tol * (1.0 + d[j]);
        }
        if (!ok && ++bad <= max_report) std::cerr << "KNN VERIFY: mismatch at point " << i << std::endl;
    }
    if (bad) {
        std::cerr << "KNN VERIFY: failed " << bad << " / " << n << " points mismatch." << std::endl;
        return false;
    }
    std::cout << "KNN VERIFY: passed - all points match brute-force." << std::endl;
    return true;
}

#ifdef WRITE_KNN_OUTPUT
void write_knn_output(knn_problem* kp) {
    POINT_TYPE* p = get_points(kp);
    unsigned int* nn = get_knearest(kp);
    unsigned int* perm = get_permutation(kp);
    std::string f = input.getParameter("output_knn_file");
    if (!output.writeKNNFile(f, p, nn, perm, kp->len_pts, _K_)) std::exit(EXIT_FAILURE);
    free(p);
    free(nn);
    free(perm);
}
#endif

}  // namespace knn
