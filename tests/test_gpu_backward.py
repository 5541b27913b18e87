"""GPU parity of the differentiable distances (the hand-written backward).

L = sum_ij w_ij * d_ij with w ~ N(0, 1) (seeded) over the FP32 squared
distances the forward returns; indices are integer and carry no gradient.

  * FP64 central finite differences, h = 1e-4 m, of L with the neighbour
    indices held fixed, on a 2,048-point sub-cloud of the uneven batch: every
    coordinate, relative error <= 1e-4 (max-norm, and per entry where the
    gradient is not tiny);
  * gather-based PyTorch autograd at full batch size: the same loss written
    as ((q[:, None] - p[idx]) ** 2).sum(-1), FP32, gradients within 1e-5 of
    the max-norm (the two sum in different orders);
  * the oracle's FP64 restatement of the backward;
  * determinism: the reference-side gradient is a segmented reduction over
    the sorted neighbour index, so two runs are bitwise identical.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"
H_FD = 1e-4  # metres


@pytest.fixture(scope="module")
def fk():
    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200.build import build
    build()
    return fk


@pytest.fixture(scope="module")
def batch():
    from flashknn_exprepo_b200 import synthetic as S
    return S.uneven_batch()


def _loss_f64(q, p, idx, w):
    """L = sum w_ij |q_i - p_idx_ij|^2 in FP64 over the valid entries."""
    valid = idx >= 0
    d = ((q[:, None, :] - p[np.where(valid, idx, 0)]) ** 2).sum(-1)
    return float((np.where(valid, w, 0.0) * d).sum())


def _central_fd(x, idx, w, q=None):
    """FP64 central differences of L w.r.t. every coordinate of x (self query:
    q is x; otherwise x is the support and q is fixed)."""
    x = x.astype(np.float64)
    g = np.zeros_like(x)
    for a in range(x.shape[0]):
        for c in range(3):
            xp = x.copy()
            xm = x.copy()
            xp[a, c] += H_FD
            xm[a, c] -= H_FD
            if q is None:
                lp, lm = _loss_f64(xp, xp, idx, w), _loss_f64(xm, xm, idx, w)
            else:
                lp, lm = _loss_f64(q, xp, idx, w), _loss_f64(q, xm, idx, w)
            g[a, c] = (lp - lm) / (2 * H_FD)
    return g


def _local_fd(x, idx, w):
    """The same central differences, evaluating only the terms of L that
    involve the perturbed point (the others cancel exactly in lp - lm)."""
    x = x.astype(np.float64)
    n, k = idx.shape
    rows_of = [[] for _ in range(n)]
    for i in range(n):
        for j in range(k):
            if idx[i, j] >= 0:
                rows_of[idx[i, j]].append(i)
    g = np.zeros_like(x)
    for a in range(n):
        rows = sorted(set(rows_of[a]) | {a})
        sub_idx = idx[rows]
        sub_w = w[rows]
        for c in range(3):
            for sign in (1.0, -1.0):
                xs = x.copy()
                xs[a, c] += sign * H_FD
                val = _loss_f64(xs[rows], xs, sub_idx, sub_w)
                g[a, c] += sign * val / (2 * H_FD)
    return g


def _subcloud(batch, count=2048):
    from flashknn_exprepo_b200 import synthetic as S
    first = batch.xyz[: batch.offsets[0]]
    return S.crop(first, count, np.random.default_rng(S.SEED))


def _masked(w, dist):
    return w * torch.isfinite(dist).to(w.dtype)


def _rel_max(got, want):
    return np.abs(got - want).max() / max(np.abs(want).max(), 1e-30)


def test_c5_finite_differences_on_2048_point_subcloud(fk, batch):
    from flashknn_exprepo_b200 import synthetic as S
    xyz = _subcloud(batch)
    n, k = len(xyz), 16
    x = torch.from_numpy(xyz).to(DEV).requires_grad_(True)
    offs = torch.tensor([n], device=DEV)
    idx, dist = fk.knn_query(k, x, offs, voxel_size=S.C4_VOXEL, num_down=2)
    w = torch.from_numpy(S.backward_weights(n, k)).to(DEV)
    (_masked(w, dist) * dist.nan_to_num(posinf=0.0)).sum().backward()
    got = x.grad.cpu().numpy().astype(np.float64)
    idx_h = idx.cpu().numpy()
    idx_fd = np.where(np.isfinite(dist.detach().cpu().numpy()), idx_h, -1)
    w64 = S.backward_weights(n, k).astype(np.float64)
    fd = _local_fd(xyz, idx_fd, w64)
    assert _rel_max(got, fd) <= 1e-4
    big = np.abs(fd) > 1e-3 * np.abs(fd).max()
    assert np.all(np.abs(got - fd)[big] <= 1e-4 * np.abs(fd)[big] + 1e-6 * np.abs(fd).max())
    # the oracle's FP64 backward agrees with the finite differences
    gq, gp = O.backward_f64(xyz, xyz, idx_fd, np.where(idx_fd >= 0, 0.0, np.inf), w64)
    assert _rel_max(gq + gp, fd) <= 1e-6


def test_local_fd_equals_full_fd_on_a_small_cloud():
    """The local evaluation above is the full central difference: check it on
    a cloud small enough to evaluate L whole for every coordinate."""
    rng = np.random.default_rng(5)
    x = rng.random((40, 3))
    idx = rng.integers(-1, 40, (40, 4))
    w = rng.standard_normal((40, 4))
    assert np.allclose(_local_fd(x, idx, w), _central_fd(x, idx, w), rtol=1e-7, atol=1e-9)


def test_c5_general_queries_fd_on_support_and_queries(fk, batch):
    from flashknn_exprepo_b200 import synthetic as S
    xyz = _subcloud(batch)
    rng = np.random.default_rng(8)
    q = (xyz[rng.choice(len(xyz), 512, replace=False)]
         + rng.normal(0, 0.01, (512, 3)).astype(np.float32))
    k = 16
    p_t = torch.from_numpy(xyz).to(DEV).requires_grad_(True)
    q_t = torch.from_numpy(q).to(DEV).requires_grad_(True)
    idx, dist = fk.knn_query(k, p_t, torch.tensor([len(xyz)], device=DEV), q_t,
                             torch.tensor([len(q)], device=DEV), voxel_size=S.C4_VOXEL)
    w = torch.from_numpy(S.backward_weights(len(q), k)).to(DEV)
    (_masked(w, dist) * dist.nan_to_num(posinf=0.0)).sum().backward()
    idx_fd = np.where(np.isfinite(dist.detach().cpu().numpy()), idx.cpu().numpy(), -1)
    w64 = w.cpu().numpy().astype(np.float64)
    gq, gp = O.backward_f64(q, xyz, idx_fd, np.where(idx_fd >= 0, 0.0, np.inf), w64)
    assert _rel_max(q_t.grad.cpu().numpy(), gq) <= 1e-5
    assert _rel_max(p_t.grad.cpu().numpy(), gp) <= 1e-5
    # FD on a sample of support coordinates (queries fixed)
    pts = rng.choice(len(xyz), 64, replace=False)
    for a in pts:
        for c in range(3):
            xp = xyz.astype(np.float64).copy()
            xm = xp.copy()
            xp[a, c] += H_FD
            xm[a, c] -= H_FD
            fd = (_loss_f64(q.astype(np.float64), xp, idx_fd, w64)
                  - _loss_f64(q.astype(np.float64), xm, idx_fd, w64)) / (2 * H_FD)
            assert abs(p_t.grad[a, c].item() - fd) <= 1e-4 * max(abs(gp).max(), 1e-30)


def test_c5_full_size_matches_gather_autograd(fk, batch):
    from flashknn_exprepo_b200 import synthetic as S
    n, k = len(batch.xyz), 16
    x = torch.from_numpy(batch.xyz).to(DEV).requires_grad_(True)
    offs = torch.from_numpy(batch.offsets).to(DEV)
    idx, dist = fk.knn_query(k, x, offs, voxel_size=S.C4_VOXEL, num_down=2)
    w = _masked(torch.from_numpy(S.backward_weights(n, k)).to(DEV), dist)
    (w * dist.nan_to_num(posinf=0.0)).sum().backward()
    ours = x.grad.clone()
    # the same loss through torch's gather and autograd
    xr = torch.from_numpy(batch.xyz).to(DEV).requires_grad_(True)
    d = ((xr[:, None, :] - xr[idx.long()]) ** 2).sum(-1)
    (w * d).sum().backward()
    ref = xr.grad
    err = ((ours - ref).abs().max() / ref.abs().max()).item()
    assert err <= 1e-5, err
    # and the forward distances equal the gathered ones up to FP32 rounding
    fin = torch.isfinite(dist)
    assert torch.allclose(dist[fin], d.detach()[fin], rtol=1e-5, atol=1e-10)


def test_backward_is_deterministic(fk, batch):
    from flashknn_exprepo_b200 import synthetic as S
    clouds = S.first_clouds(batch, 4)
    x = torch.from_numpy(clouds.xyz).to(DEV)
    offs = torch.from_numpy(clouds.offsets).to(DEV)
    idx, dist = fk.ops.knn_offsets(x, offs, 16, S.C4_VOXEL, 2)
    g = torch.from_numpy(S.backward_weights(len(clouds.xyz), 16)).to(DEV)
    g = _masked(g, dist)
    runs = []
    for _ in range(3):
        gq = torch.empty_like(x)
        gp = torch.empty_like(x)
        fk.ops.backward(x, x, idx, dist, g, grad_q=gq, grad_p=gp)
        runs.append((gq.cpu().numpy().view(np.uint32), gp.cpu().numpy().view(np.uint32)))
    for gq, gp in runs[1:]:
        assert np.array_equal(gq, runs[0][0]) and np.array_equal(gp, runs[0][1])


def test_backward_ignores_padding_entries(fk):
    # a point alone in its neighbourhood: K-1 padding slots (self, +inf)
    xyz = np.array([[0.5, 0.5, 0.5], [0.9, 0.9, 0.9], [0.905, 0.9, 0.9]], np.float32)
    x = torch.from_numpy(xyz).to(DEV).requires_grad_(True)
    idx, dist = fk.knn_query(4, x, torch.tensor([3], device=DEV), voxel_size=0.01, num_down=1)
    assert torch.isinf(dist).any()
    (dist.nan_to_num(posinf=0.0)).sum().backward()
    g = x.grad.cpu().numpy()
    assert np.all(np.isfinite(g))
    assert np.all(g[0] == 0)
    # the pair (1, 2): d = |x1 - x2|^2 counted twice (1->2 and 2->1)
    want = 4 * (xyz[1] - xyz[2]).astype(np.float64)
    assert np.allclose(g[1], want, rtol=1e-5) and np.allclose(g[2], -want, rtol=1e-5)


def test_hub_points_with_long_segments(fk):
    """Exact duplicates make the lowest-index copies the neighbours of every
    copy (ties break by lower index), so a few support points collect
    hundreds of entries: the warp-cooperative path of the segmented sum."""
    rng = np.random.default_rng(12)
    base = rng.random((2000, 3), dtype=np.float32)
    hub = np.repeat(base[:3], 150, axis=0)          # three clusters of 150 copies
    xyz = np.concatenate([base[3:], hub])
    rng.shuffle(xyz)
    n, k = len(xyz), 16
    x = torch.from_numpy(xyz).to(DEV)
    offs = torch.tensor([n], device=DEV)
    idx, dist = fk.ops.knn_offsets(x, offs, k, 0.03, 2)
    counts = np.bincount(idx.cpu().numpy().ravel(), minlength=n)
    assert counts.max() > 100
    g = torch.from_numpy(np.random.default_rng(3).standard_normal((n, k)).astype(np.float32))
    g = _masked(g.to(DEV), dist)
    outs = []
    for _ in range(2):
        gq = torch.empty_like(x)
        gp = torch.empty_like(x)
        fk.ops.backward(x, x, idx, dist, g, grad_q=gq, grad_p=gp)
        outs.append((gq.cpu().numpy(), gp.cpu().numpy()))
    assert np.array_equal(outs[0][1].view(np.uint32), outs[1][1].view(np.uint32))
    wq, wp = O.backward_f64(xyz, xyz, idx.cpu().numpy(), dist.cpu().numpy(),
                            g.cpu().numpy().astype(np.float64))
    assert _rel_max(outs[0][0], wq) <= 1e-5
    assert _rel_max(outs[0][1], wp) <= 1e-5


@pytest.mark.parametrize("k", [1, 3, 7, 12, 24, 33, 64])
def test_backward_list_lengths(fk, k):
    """Every row length: entry e = i*K+j maps back to its query row by a
    multiply-shift division (exact for every K, power of two or not), and
    K not a multiple of 4 takes the scalar row loads.  Against the oracle's
    FP64 backward, and bitwise identical run to run."""
    rng = np.random.default_rng(100 + k)
    xyz = rng.random((6000, 3), dtype=np.float32)
    n = len(xyz)
    x = torch.from_numpy(xyz).to(DEV)
    offs = torch.tensor([n], device=DEV)
    idx, dist = fk.ops.knn_offsets(x, offs, k, 0.02, 2)
    g = torch.from_numpy(rng.standard_normal((n, k)).astype(np.float32)).to(DEV)
    g = _masked(g, dist)
    outs = []
    for _ in range(2):
        gq = torch.empty_like(x)
        gp = torch.empty_like(x)
        fk.ops.backward(x, x, idx, dist, g, grad_q=gq, grad_p=gp)
        outs.append((gq.cpu().numpy(), gp.cpu().numpy()))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    wq, wp = O.backward_f64(xyz, xyz, idx.cpu().numpy(), dist.cpu().numpy(),
                            g.cpu().numpy().astype(np.float64))
    assert _rel_max(outs[0][0], wq) <= 1e-5
    assert _rel_max(outs[0][1], wp) <= 1e-5


def test_buckets_beyond_the_stage_and_a_point_beyond_it(fk):
    """Arbitrary neighbour tables (the backward takes any idx): one point
    named by 20,000 rows (more entries than a bucket's whole shared-memory
    stage: summed by a warp streaming the runs) and forty points named by 500
    rows each (one bucket holding more than the stage: several point ranges),
    the rest random.  Against the oracle's FP64 backward, bitwise identical
    run to run."""
    rng = np.random.default_rng(21)
    m, n, k = 40000, 30000, 8
    q = rng.random((m, 3), dtype=np.float32)
    p = rng.random((n, 3), dtype=np.float32)
    idx = rng.integers(100, n, size=(m, k)).astype(np.int32)
    idx[:20000, 0] = 0                                   # the hub
    idx[20000:, 1] = 1 + (np.arange(m - 20000) % 40)     # 40 points x 500 rows
    dist = ((q[:, None, :] - p[idx]) ** 2).sum(-1).astype(np.float32)
    dist[rng.random((m, k)) < 0.01] = np.inf             # some padding entries
    g = rng.standard_normal((m, k)).astype(np.float32)
    Q, P, I, D, G = (torch.from_numpy(a).to(DEV) for a in (q, p, idx, dist, g))
    outs = []
    for _ in range(2):
        gq = torch.empty_like(Q)
        gp = torch.empty_like(P)
        fk.ops.backward(Q, P, I, D, G, grad_q=gq, grad_p=gp)
        outs.append((gq.cpu().numpy(), gp.cpu().numpy()))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    wq, wp = O.backward_f64(q, p, idx, dist, g.astype(np.float64))
    assert _rel_max(outs[0][0], wq) <= 1e-5
    # the hub's gradient is a sequential FP32 sum of 20,000 terms: its
    # rounding error grows like sqrt(20000) * 2^-24 of the result
    assert _rel_max(outs[0][1], wp) <= 5e-5
