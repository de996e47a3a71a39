"""The FP64 fixed points bench.py computes with PyTorch to report each
result's max and L1 error, held to the oracle's own converged FP64 solutions
(CPU tensors; the same code runs on the GPU in the bench)."""
import numpy as np
import pytest
import torch

import bench


class _Arr:
    def __init__(self, a):
        self.a = a

    def to_numpy(self):
        return self.a


class _CSR:
    """The (rowptr, col, third) shape of the library's device CSR objects."""

    def __init__(self, rp, col, od):
        self.rowptr, self.col, self.third = _Arr(rp), _Arr(col), _Arr(od)


def test_pagerank_fixed_point_matches_oracle(O):
    rp, col, od = O.rmat_graph(10, 8, seed=3)
    m = len(rp) - 1
    ref, _, _ = O.pr_f64(rp, col, od, tol=1e-15, max_iter=3000)
    start, _, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=100)
    x, it, delta = bench.fp64_fixed_point(torch, _CSR(rp, col, od), m, torch.from_numpy(start))
    assert delta < 1e-13 and it < 400
    np.testing.assert_allclose(x.numpy(), ref, rtol=0, atol=1e-12)
    err = bench.errors_vs(x, torch.from_numpy(start))
    assert err["max_error_vs_fp64_fixed_point"] <= err["l1_error_vs_fp64_fixed_point"]
    assert err["l1_error_vs_fp64_fixed_point"] == pytest.approx(np.abs(start - ref).sum(), rel=1e-9)


def test_ppr_fixed_point_matches_oracle(O):
    rp, col, od = O.rmat_graph(10, 8, seed=4)
    m = len(rp) - 1
    seeds = O.uniform_int(6, 9, m)
    seeds[1] = seeds[0]  # two vectors with one seed
    ref, _ = O.ppr_f64(rp, col, od, seeds, tol=1e-15, max_iter=3000)
    start, _ = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    x = bench.ppr_fp64_fixed_point(torch, _CSR(rp, col, od), m, seeds,
                                   torch.from_numpy(start.astype(np.float32)))
    np.testing.assert_allclose(x.numpy(), ref, rtol=0, atol=1e-12)


def test_batch_fixed_point_matches_per_graph_oracle(O):
    """A block-diagonal batch with each graph's own teleport (1 - d) / m_g:
    the batch's fixed point is every graph's own fixed point."""
    rp, col, od, voff = O.multigraph(4, 100, 2000, seed=2)
    M = len(rp) - 1
    m_g = np.diff(voff).astype(np.int64)
    base = np.repeat((1.0 - float(np.float32(0.85))) / m_g, m_g)
    start = np.repeat(1.0 / m_g, m_g).astype(np.float32)
    x, it, delta = bench.fp64_fixed_point(torch, _CSR(rp, col, od), M, torch.from_numpy(start),
                                          base=torch.from_numpy(base))
    assert delta < 1e-13
    for g in range(len(voff) - 1):
        a, b = voff[g], voff[g + 1]
        e0, e1 = rp[a], rp[b]
        ref, _, _ = O.pr_f64(rp[a:b + 1] - e0, col[e0:e1] - a, od[a:b], tol=1e-15, max_iter=3000)
        np.testing.assert_allclose(x.numpy()[a:b], ref, rtol=0, atol=1e-12)
