"""Learned neighbour budget: the device MLP against a PyTorch FP32 reference of the
same network, and learned-K moving-mesh steps against plain fixed-K steps (the
mesh, and therefore every step, must be identical bit for bit)."""
import numpy as np
import pytest

from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _unpack(w):
    if not isinstance(w, torch.Tensor):
        w = torch.as_tensor(np.asarray(w, np.float32))
    return (w[0:256].reshape(32, 8), w[256:288], w[288:1312].reshape(32, 32), w[1312:1344],
            w[1344:1536].reshape(6, 32), w[1536:1542])


def _bf(t):
    """Rounds to BF16 in the forward pass and passes the gradient straight through."""
    return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()


def torch_mlp(w, x):
    """The network with the kernel's rounding points: BF16 inputs, weights and
    hidden activations; FP32 accumulation, biases and logits."""
    W1, b1, W2, b2, W3, b3 = _unpack(w)
    x = _bf(torch.as_tensor(np.asarray(x, np.float32)))
    h1 = _bf(torch.nn.functional.gelu(x @ _bf(W1).T + b1))
    h2 = _bf(torch.nn.functional.gelu(h1 @ _bf(W2).T + b2))
    return h2 @ _bf(W3).T + b3


def _features(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.normal(0.0, 1.0, (n, 8)).astype(np.float32)
    f[:, 5] = (rng.random(n) < 0.1).astype(np.float32)
    return f


def _trained_like_weights(ctx, seed):
    rng = np.random.default_rng(seed)
    w = ctx.kbudget_weights()
    w = (w + rng.normal(0.0, 0.05, w.shape)).astype(np.float32)
    w[1536:1542] = rng.normal(0.0, 0.5, 6)  # output biases: uneven class priors
    return ctx.kbudget_weights(w)


@pytest.mark.parametrize("dim", [2, 3])
def test_mlp_forward_matches_torch(dim):
    feat = _features(5000, 1)
    with Context(dim=dim, k=190 if dim == 3 else 48) as ctx:
        w = _trained_like_weights(ctx, 2)
        logits, kq = ctx.mlp_forward(feat)
        from proteusgpu_b200 import _lib
        classes = (np.zeros(6, np.int32))
        _lib.load().pgpu_kbudget_classes(dim, classes.ctypes.data)
    ref = torch_mlp(w, feat).detach().numpy()
    # same rounding points and FP32 accumulation; summation order differs
    assert np.abs(logits - ref).max() <= 2e-3 * max(1.0, np.abs(ref).max())
    p = np.exp(ref - ref.max(1, keepdims=True))
    cum = np.cumsum(p / p.sum(1, keepdims=True), axis=1)
    want = classes[np.argmax(cum >= 0.99, axis=1)]
    decided = np.abs(cum - 0.99).min(1) > 1e-4  # rows not on the quantile's edge
    assert np.array_equal(kq[decided], want[decided])
    assert decided.mean() > 0.99


def test_mlp_gradient_matches_torch_autograd():
    feat = _features(4096, 3)
    labels = np.random.default_rng(4).integers(0, 6, len(feat)).astype(np.int32)
    with Context(dim=3, k=190) as ctx:
        w = _trained_like_weights(ctx, 5)
        g, loss = ctx.mlp_grad(feat, labels)
    wt = torch.tensor(w, requires_grad=True)
    logits = torch_mlp(wt, feat)
    ref_loss = torch.nn.functional.cross_entropy(logits, torch.as_tensor(labels, dtype=torch.long))
    ref_loss.backward()
    gr = wt.grad.numpy()
    assert abs(loss - ref_loss.item()) <= 1e-4 * abs(ref_loss.item())
    # the kernel rounds the backward deltas to BF16 for the tensor cores
    for a, b in [(0, 256), (256, 288), (288, 1312), (1312, 1344), (1344, 1536), (1536, 1542)]:
        assert np.linalg.norm(g[a:b] - gr[a:b]) <= 2e-2 * np.linalg.norm(gr[a:b]) + 1e-7


def _sim(ic, k, buff, steps, kbudget, precision="fp64", train_steps=2, quantile=0.99):
    with Context(dim=ic.dim, k=k, buff=buff, flux="physical", gamma=ic.gamma, precision=precision) as ctx:
        if kbudget:
            ctx.kbudget_enable(train_steps=train_steps, iters_per_step=48, quantile=quantile, seed=3)
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        info = []
        for _ in range(steps):
            ctx.sim_step(0.3)
            if kbudget:
                info.append(ctx.kbudget_stats())
        mesh = ctx.download_mesh()
        x, mass, mom, en = ctx.sim_get()
        st = ctx.stats()
    return x, mass, mom, en, mesh, info, st


def _same(a, b):
    for u, v in zip(a[:4], b[:4]):
        assert np.array_equal(u, v)
    ma, mb = a[4], b[4]
    assert np.array_equal(ma.face_counts, mb.face_counts) and np.array_equal(ma.neighbor, mb.neighbor)
    assert np.array_equal(ma.area, mb.area) and np.array_equal(ma.volumes, mb.volumes)
    assert np.array_equal(ma.status, mb.status) and np.array_equal(ma.cert_k, mb.cert_k)


def test_learned_k_steps_equal_plain_steps_3d():
    ic = ics.sedov_3d(n=30000, seed=6)
    plain = _sim(ic, 190, 0.1, 6, False)
    learned = _sim(ic, 190, 0.1, 6, True)
    _same(learned, plain)
    info = learned[5]
    assert info[-1]["active"] == 1 and info[-1]["steps_trained"] == 2
    assert info[-1]["cells"] == len(ic.pos)
    # the proposal saves work: mean K well below the plain 190, few cells recomputed
    assert info[-1]["mean_k"] < 110
    assert info[-1]["misses"] < 0.05 * len(ic.pos)


def test_learned_k_with_fp32_clipping_equals_plain_fp64():
    ic = ics.sedov_3d(n=20000, seed=9)
    plain = _sim(ic, 190, 0.1, 5, False)
    fast = _sim(ic, 190, 0.1, 5, True, precision="fp32")
    _same(fast, plain)


def test_learned_k_2d_kelvin_helmholtz():
    ic = ics.kh_2d(n_side=96, seed=3)
    plain = _sim(ic, 48, 0.08, 6, False)
    learned = _sim(ic, 48, 0.08, 6, True, train_steps=3)
    _same(learned, plain)
    assert learned[5][-1]["mean_k"] < 40


def test_every_proposal_rejected_still_gives_the_plain_mesh():
    """Quantile 1e-6: the smallest class almost everywhere, so most cells miss and
    are recomputed at the plain K -- the result must not change."""
    ic = ics.sedov_3d(n=15000, seed=10)
    plain = _sim(ic, 190, 0.1, 4, False)
    starved = _sim(ic, 190, 0.1, 4, True, quantile=1e-6)
    _same(starved, plain)
    assert starved[5][-1]["misses"] > 0


def test_learned_k_with_thread_per_query_knn():
    """Per-query K from 32 to 128 split between the thread kernel (K <= 64) and
    the warp kernel (the rest) in one search: the steps still equal the plain ones."""
    ic = ics.sedov_3d(n=20000, seed=14)
    plain = _sim(ic, 190, 0.1, 4, False)
    with Context(dim=3, k=190, buff=0.1, flux="physical", gamma=ic.gamma, precision="fp32") as ctx:
        ctx.set_tuning(knn_thread=64)
        ctx.kbudget_enable(train_steps=2, iters_per_step=48, quantile=0.99, seed=3)
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        for _ in range(4):
            ctx.sim_step(0.3)
        mesh = ctx.download_mesh()
        got = ctx.sim_get() + (mesh,)
    _same(got, plain)


def test_clustered_walk_forms_identical_without_failures():
    """Clustered points: cells beside the clumps need the grid walk.  The walk starts
    from the same list prefix in every form, so learned-K + FP32 steps still equal the
    plain FP64 steps bit for bit, and no cell fails (none collects more than the
    reference's 96 vertices on the way)."""
    ic = ics.clustered_3d(n=150000, seed=5)
    plain = _sim(ic, 190, 0.1, 4, False)
    fast = _sim(ic, 190, 0.1, 4, True, precision="fp32")
    _same(fast, plain)
    for st in (plain[6], fast[6]):
        assert st["pruned_cells"] > 0
        assert st["failed_cells"] == 0
