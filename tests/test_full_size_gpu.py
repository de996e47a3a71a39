"""Parity at the benchmark sizes (minutes of CPU work on the host's cores).

The graphs are generated on the GPU (bit-identical to the oracle's
generators, tests/test_gen_gpu.py and tests/test_multi_gpu.py) and copied to
the host for the oracle:
  * PageRank on RMAT scale 24 (16.8M vertices, 263M edges), tol 1e-6: the
    reference's sweep count within one, every vertex within 1e-6 plus the
    reference's own float error, and the FP64 oracle's L1 error within the
    metric's 1e-5;
  * the 512-graph batch: a sample of its graphs (the largest, the smallest and
    some in between) against the oracle, each solved inside the full batch;
  * batched personalized PageRank on RMAT scale 22 with 8 seeds against the
    FP64 oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rmat24_pagerank_full_size(G, O):
    """Both sweep forms at full size: the exact-order layout, and the blocked
    layout that AUTO solves in the blocked form at this size (and, from a
    non-finite score, in the exact form)."""
    csr = G.gen_rmat(24, 16, seed=1)
    rp, col, od = csr.rowptr.to_numpy(), csr.col.to_numpy(), csr.third.to_numpy()
    m = csr.m
    bad = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    bad[7] = np.inf
    with G.Graph(csr.rowptr, csr.col, csr.third, m=m, nnz=csr.nnz) as g:
        s, st = g.pagerank(tol=1e-6, max_iter=100)
        s_bad, st_bad = g.pagerank(bad.copy(), tol=1e-6, max_iter=3)
    with G.Graph(csr.rowptr, csr.col, csr.third, m=m, nnz=csr.nnz, blocked=True) as g:
        sb, stb = g.pagerank(tol=1e-6, max_iter=100)
        sb_bad, stb_bad = g.pagerank(bad.copy(), tol=1e-6, max_iter=3)
    csr.close()
    assert stb_bad.iterations == st_bad.iterations
    assert np.array_equal(np.isnan(sb_bad), np.isnan(s_bad))
    assert np.array_equal(sb_bad[~np.isnan(sb_bad)], s_bad[~np.isnan(s_bad)])
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=100)
    fix, _, _ = O.pr_f64(rp, col, od, tol=1e-13, max_iter=400)
    for got, n in ((s, st.iterations), (sb, stb.iterations)):
        assert abs(n - ref_it) <= 1
        s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=n)
        assert np.all(np.abs(got - ref) <= 1e-6 + np.abs(ref - s64))
        _, l1 = O.err_vs_f64(got, fix)
        assert l1 <= 1e-5


def test_multigraph_512_sample_full_size(G, O):
    A, voff = G.gen_multigraph(512, 1000, 500000, seed=1)
    with G.MultiGraph(A.rowptr, A.col, A.third, voff, nnz=A.nnz) as mg:
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=200)
    rp, col, od = A.rowptr.to_numpy(), A.col.to_numpy(), A.third.to_numpy()
    A.close()
    sizes = np.diff(voff)
    sample = sorted({int(np.argmax(sizes)), int(np.argmin(sizes)),
                     *np.random.default_rng(3).choice(512, 6, replace=False).tolist()})
    for g in sample:
        a, b = int(voff[g]), int(voff[g + 1])
        e0, e1 = int(rp[a]), int(rp[b])
        lrp, lcol, lod = rp[a:b + 1] - e0, col[e0:e1] - a, od[a:b]
        ref, ref_it, _ = O.pr_plain_f32(lrp, lcol, lod, tol=1e-6, max_iter=200)
        assert abs(int(iters[g]) - ref_it) <= 1, g
        s64, _, _ = O.pr_f64(lrp, lcol, lod, tol=0.0, max_iter=int(iters[g]))
        assert np.all(np.abs(s[a:b] - ref) <= 1e-6 + np.abs(ref - s64)), g


def test_ppr_rmat22_full_size(G, O):
    csr = G.gen_rmat(22, 16, seed=1)
    rp, col, od = csr.rowptr.to_numpy(), csr.col.to_numpy(), csr.third.to_numpy()
    seeds = np.random.default_rng(22).integers(0, csr.m, 8).astype(np.int32)
    with G.Graph(csr.rowptr, csr.col, csr.third, m=csr.m, nnz=csr.nnz, batched=True) as g:
        x, it, st = g.ppr(seeds, tol=1e-6, max_iter=100)
    csr.close()
    ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    assert np.all(np.abs(x - ref).sum(axis=0) <= 1e-5)
    assert np.all(np.abs(it - ref_it) <= 1)
