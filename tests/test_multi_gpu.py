"""Uneven multi-graph batch on the GPU through the C ABI.

Each graph of a batch must come out exactly as the single-graph solver
computes it alone (bit-identical scores, the same sweep count), and within
the plain path's bar of the reference's OpenMP PRSolver restated in the
oracle: 1e-6 absolute per vertex, sweeps within one.  The GPU generator must
reproduce the oracle's generator bit for bit.
"""
import numpy as np
import pytest

from graphs import erdos_renyi

pytestmark = pytest.mark.gpu


def local(rp, col, od, voff, g):
    """Graph g of a block-diagonal batch as its own CSR (local vertex ids)."""
    a, b = int(voff[g]), int(voff[g + 1])
    e0, e1 = int(rp[a]), int(rp[b])
    return (rp[a:b + 1] - e0).astype(np.int32), (col[e0:e1] - a).astype(np.int32), od[a:b]


def concat(graphs):
    """Block-diagonal batch of local CSRs -> (rowptr, col, outdeg, voff)."""
    rps, cols, ods, voff, e, v = [], [], [], [0], 0, 0
    for rp, col, od in graphs:
        rps.append(rp[:-1].astype(np.int64) + e)
        cols.append(col.astype(np.int64) + v)
        ods.append(od)
        e += int(rp[-1])
        v += len(rp) - 1
        voff.append(v)
    rp = np.concatenate(rps + [np.array([e])]).astype(np.int32)
    return rp, np.concatenate(cols).astype(np.int32), np.concatenate(ods).astype(np.int32), \
        np.array(voff, np.int32)


@pytest.fixture(scope="module")
def batch(O):
    # 12 graphs, sizes log-uniform in [200, 30000]; the Chung-Lu ones have
    # hubs of several thousand in-edges (chunked rows).
    return O.multigraph(12, 200, 30000, seed=4)


def test_generator_identical(G, O):
    rp, col, od, voff = O.multigraph(9, 100, 5000, seed=3)
    A, gv = G.gen_multigraph(9, 100, 5000, seed=3)
    assert np.array_equal(gv, voff)
    assert A.nnz == len(col)
    assert np.array_equal(A.rowptr.to_numpy(), rp)
    assert np.array_equal(A.col.to_numpy(), col)
    assert np.array_equal(A.third.to_numpy(), od)
    A.close()


@pytest.mark.parametrize("tol,max_iter", [(1e-6, 100), (1e-4, 100), (1e-7, 12)])
def test_batch_matches_single_graph_solves(G, O, batch, tol, max_iter):
    rp, col, od, voff = batch
    n = len(voff) - 1
    with G.MultiGraph(rp, col, od, voff) as mg:
        info = mg.info()
        s, iters, res, st = mg.pagerank(tol=tol, max_iter=max_iter)
    assert info["n_graphs"] == n and info["nnz"] == len(col)
    assert st.iterations == iters.max()
    for g in range(n):
        lrp, lcol, lod = local(rp, col, od, voff, g)
        with G.Graph(lrp, lcol, lod) as one:
            s1, st1 = one.pagerank(tol=tol, max_iter=max_iter)
        a, b = voff[g], voff[g + 1]
        assert iters[g] == st1.iterations, g
        assert np.array_equal(s[a:b], s1), g
        assert res[g] == pytest.approx(st1.residual, rel=1e-12, abs=1e-300)


def test_batch_matches_reference(G, O, batch):
    # chunk_min 512 / chunk 256: the Chung-Lu hubs become multi-chunk rows
    rp, col, od, voff = batch
    n = len(voff) - 1
    lays = [{"chunk_min": 512, "chunk": 256}] * n
    with G.MultiGraph(rp, col, od, voff, layouts=lays) as mg:
        s, iters, res, _ = mg.pagerank(tol=1e-6, max_iter=100)
    hubs = 0
    for g in range(n):
        lrp, lcol, lod = local(rp, col, od, voff, g)
        hubs += int(np.diff(lrp).max() > 512)
        ref, ref_it, _ = O.pr_plain_f32(lrp, lcol, lod, tol=1e-6, max_iter=100)
        a, b = voff[g], voff[g + 1]
        assert abs(int(iters[g]) - ref_it) <= 1, g
        s64, _, _ = O.pr_f64(lrp, lcol, lod, tol=0.0, max_iter=int(iters[g]))
        assert np.all(np.abs(s[a:b] - ref) <= 1e-6 + np.abs(ref - s64)), g
    assert hubs > 0  # chunked rows were exercised


def test_per_graph_bins(G, O, batch):
    # Each graph with its own bins gives what the single-graph solver gives
    # with the same layout options.
    rp, col, od, voff = batch
    n = len(voff) - 1
    lays = [{"sell_max": (8, 16, 32, 64)[g % 4], "chunk_min": (512, 1024, 4096)[g % 3],
             "chunk": (128, 512, 4096)[g % 3]} for g in range(n)]
    with G.MultiGraph(rp, col, od, voff, layouts=lays) as mg:
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=60)
    for g in range(n):
        lrp, lcol, lod = local(rp, col, od, voff, g)
        with G.Graph(lrp, lcol, lod, **lays[g]) as one:
            s1, st1 = one.pagerank(tol=1e-6, max_iter=60)
        assert iters[g] == st1.iterations
        assert np.array_equal(s[voff[g]:voff[g + 1]], s1), g


def test_edge_cases(G, O):
    # empty graph, one vertex, edge-free graph, a normal graph, a star hub
    empty = (np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    one = (np.zeros(2, np.int32), np.zeros(0, np.int32), np.zeros(1, np.int32))
    bare = (np.zeros(301, np.int32), np.zeros(0, np.int32), np.zeros(300, np.int32))
    er = erdos_renyi(5000, 6, seed=9)
    m = 9000
    src = np.arange(1, m)
    hub_rp = np.array([0, m - 1] + [m - 1] * (m - 1), np.int32)
    hub = (hub_rp, src.astype(np.int32), np.concatenate([[0], np.ones(m - 1)]).astype(np.int32))
    parts = [empty, one, er, bare, hub, empty]
    rp, col, od, voff = concat(parts)
    for tol, mi in ((1e-6, 50), (0.0, 7), (1e-6, 0)):
        with G.MultiGraph(rp, col, od, voff) as mg:
            s, iters, res, _ = mg.pagerank(tol=tol, max_iter=mi)
        for g, (lrp, lcol, lod) in enumerate(parts):
            a, b = voff[g], voff[g + 1]
            with np.errstate(divide="ignore"):
                ref, ref_it, _ = O.pr_plain_f32(lrp, lcol, lod, tol=tol, max_iter=mi)
            # an empty graph counts the reference's empty sweeps too
            assert iters[g] == ref_it, (g, tol, mi)
            if b == a:
                assert res[g] == 0.0
                continue
            # the hub's 8999-term sequential float sum in the reference is
            # itself off from the exact sum: bound by its FP64 distance
            s64, _, _ = O.pr_f64(lrp, lcol, lod, tol=0.0, max_iter=ref_it)
            assert np.all(np.abs(s[a:b] - ref) <= 1e-6 + np.abs(ref - s64)), (g, tol, mi)


def test_rejects_edges_across_graphs(G):
    rp, col, od = erdos_renyi(100, 4, seed=1)
    voff = np.array([0, 50, 100], np.int32)  # ER edges cross the cut
    with pytest.raises(G.GprError) as e:
        G.MultiGraph(rp, col, od, voff)
    assert e.value.status == G.GPR_EINVAL


def test_bf16_mixed_form(G, O, batch):
    rp, col, od, voff = batch
    with G.MultiGraph(rp, col, od, voff) as mg:
        s32, it32, _, _ = mg.pagerank(tol=1e-6, max_iter=200)
        sbf, itbf, _, st = mg.pagerank(tol=1e-6, max_iter=200, precision=G.PREC_BF16)
    assert st.refine_iterations > 0
    for g in range(len(voff) - 1):
        lrp, lcol, lod = local(rp, col, od, voff, g)
        s64, _, _ = O.pr_f64(lrp, lcol, lod)
        a, b = voff[g], voff[g + 1]
        _, l1_32 = O.err_vs_f64(s32[a:b], s64)
        _, l1_bf = O.err_vs_f64(sbf[a:b], s64)
        # both refined to the same tolerance: within the L1 error bar
        assert l1_32 <= 1e-5 and l1_bf <= 1e-5, (g, l1_32, l1_bf)


def test_barrier_timeout_is_reported(G, O):
    rp, col, od, voff = O.multigraph(4, 100, 2000, seed=2)
    with G.MultiGraph(rp, col, od, voff) as mg:
        o = G.options(tol=1e-6, max_iter=20, timeout_s=0.5)
        o.reserved[0] = 1
        with pytest.raises(G.GprError) as e:
            mg.pagerank(opts=o)
        assert e.value.status == G.GPR_ETIMEOUT
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=20)  # still usable
        assert iters.min() > 0


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_graph_loop_matches_persistent(G, O, batch, prec):
    """GPR_LOOP_GRAPH runs one sweep per launch inside a CUDA-graph while
    loop (the last CTA to finish a sweep closes it, no CTA waits for another);
    the sweep code is the persistent kernel's, so scores, per-graph sweep
    counts and residuals are bit-identical."""
    rp, col, od, voff = batch
    p = G.PREC_BF16 if prec == "bf16" else G.PREC_FP32
    with G.MultiGraph(rp, col, od, voff) as mg:
        s0, it0, r0, st0 = mg.pagerank(tol=1e-6, max_iter=100, precision=p, loop=G.LOOP_PERSISTENT)
        s1, it1, r1, st1 = mg.pagerank(tol=1e-6, max_iter=100, precision=p, loop=G.LOOP_GRAPH)
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_array_equal(it0, it1)
    np.testing.assert_array_equal(r0, r1)
    assert st1.iterations == st0.iterations
    assert st1.gpu_launches > st0.gpu_launches  # one launch per sweep


def test_graph_loop_caps_at_max_iter(G, O, batch):
    rp, col, od, voff = batch
    with G.MultiGraph(rp, col, od, voff) as mg:
        s1, it1, _, st1 = mg.pagerank(tol=0.0, max_iter=6, loop=G.LOOP_GRAPH)
        s0, it0, _, st0 = mg.pagerank(tol=0.0, max_iter=6)
    assert st1.iterations == 6 and it1.max() == 6
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_array_equal(it0, it1)
