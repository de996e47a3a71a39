"""PageRank on the GPU through the C ABI, checked against the oracle.

Tolerances (the bar this path is held to):
  * per-vertex |gpu - reference OpenMP| <= 1e-6 absolute, iteration count
    within one sweep (the reference runs float sums in row order; long rows
    here are summed as a tree);
  * graphs whose rows all have at most 64 in-edges are computed with the
    reference's float operations in the reference's order: bit-identical.
"""
import numpy as np
import pytest

from graphs import degree_ladder, erdos_renyi, star

pytestmark = pytest.mark.gpu

ABS_TOL = 1e-6


def solve(G, rp, col, od, **kw):
    with G.Graph(rp, col, od) as g:
        s, st = g.pagerank(**kw)
        return s, st, g.residuals(), g.layout()


def test_rmat_s16_matches_reference(G, O):
    # RMAT scale 16, edge factor 16, (0.57, 0.19, 0.19), tol 1e-4, <= 100 sweeps.
    rp, col, od = O.rmat_graph(16, 16, seed=1)
    ref, ref_it, ref_hist = O.pr_plain_f32(rp, col, od, tol=1e-4, max_iter=100)
    s, st, hist, lay = solve(G, rp, col, od, tol=1e-4, max_iter=100)
    assert lay["n_slices"] > 0
    assert abs(st.iterations - ref_it) <= 1
    assert np.abs(s - ref).max() <= ABS_TOL
    s64, _, _ = O.pr_f64(rp, col, od)
    mx_g, l1_g = O.err_vs_f64(s, s64)
    mx_r, l1_r = O.err_vs_f64(ref, s64)
    assert l1_g <= 1.05 * l1_r + 1e-9 and mx_g <= 1.05 * mx_r + 1e-9


def test_short_rows_bit_identical(G, O):
    rp, col, od = erdos_renyi(20000, 8, seed=3)
    assert np.diff(rp).max() <= 64
    ref, ref_it, ref_hist = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=100)
    s, st, hist, lay = solve(G, rp, col, od, tol=1e-6, max_iter=100)
    assert lay["n_long"] == 0 and lay["n_slices"] > 0
    assert st.iterations == ref_it
    assert np.array_equal(s, ref)
    np.testing.assert_allclose(hist, ref_hist, rtol=1e-12)


@pytest.mark.parametrize("maker", [star, degree_ladder])
@pytest.mark.parametrize("variant", list(range(8)))
def test_long_rows_and_bins(G, O, maker, variant):
    # The tolerance sits well above the float rounding floor of the L1
    # residual (about m * ulp(score) ~ 1e-7 here), where the sweep count is
    # decided by the arithmetic rather than by noise.
    # A hub with 1e5 in-edges carries a score near 0.3; the reference's own
    # sequential float sum is then off by ~1e-5 from the exact sum, so each
    # vertex may deviate from the reference by 1e-6 plus the reference's own
    # distance to an FP64 run of the same number of sweeps.
    rp, col, od = maker()
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-5, max_iter=60)
    with G.Graph(rp, col, od, chunk=512, chunk_min=1024) as g:
        lay = g.layout()
        s, st = g.pagerank(tol=1e-5, max_iter=60, variant=variant)
    assert lay["n_long"] > 0 and lay["n_chunks"] > lay["n_long"]
    assert abs(st.iterations - ref_it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=st.iterations)
    assert np.all(np.abs(s - ref) <= ABS_TOL + np.abs(ref - s64))
    assert np.abs(s - s64).max() <= np.abs(ref - s64).max() + ABS_TOL


def test_loop_modes_identical(G, O):
    rp, col, od = O.rmat_graph(14, 8, seed=5)
    a, sa, _, _ = solve(G, rp, col, od, tol=1e-6, max_iter=50, loop=G.LOOP_PERSISTENT)
    b, sb, _, _ = solve(G, rp, col, od, tol=1e-6, max_iter=50, loop=G.LOOP_GRAPH)
    assert sa.iterations == sb.iterations
    assert np.array_equal(a, b)


def test_deterministic_and_reusable(G, O):
    rp, col, od = O.rmat_graph(13, 16, seed=9)
    with G.Graph(rp, col, od) as g:
        a, sa = g.pagerank(tol=1e-6, max_iter=40)
        b, sb = g.pagerank(tol=1e-6, max_iter=40)
    assert np.array_equal(a, b) and sa.iterations == sb.iterations


def test_unconverged_runs_max_iter(G, O):
    rp, col, od = O.rmat_graph(12, 16, seed=2)
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=0.0, max_iter=7)
    s, st, hist, _ = solve(G, rp, col, od, tol=0.0, max_iter=7)
    assert st.iterations == ref_it == 7 and len(hist) == 7
    assert np.abs(s - ref).max() <= ABS_TOL


def test_warm_start_scores(G, O):
    rp, col, od = erdos_renyi(5000, 6, seed=11)
    init = np.random.default_rng(1).random(5000).astype(np.float32) / 5000
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, scores=init, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od) as g:
        s = init.copy()
        _, st = g.pagerank(s, tol=1e-6, max_iter=100)
    assert st.iterations == ref_it and np.array_equal(s, ref)


def test_device_scores_in_place(G, O):
    torch = pytest.importorskip("torch")
    rp, col, od = O.rmat_graph(12, 8, seed=4)
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-5, max_iter=100)
    m = len(rp) - 1
    d = torch.full((m,), 1.0 / m, dtype=torch.float32, device="cuda")
    with G.Graph(rp, col, od) as g:
        _, st = g.pagerank(d, tol=1e-5, max_iter=100)
    assert abs(st.iterations - ref_it) <= 1
    assert np.abs(d.cpu().numpy() - ref).max() <= ABS_TOL


@pytest.mark.filterwarnings("ignore:divide by zero")
@pytest.mark.parametrize("tol,max_iter", [(1e-3, 30), (0.0, 7), (1e-3, 0)])
def test_empty_graph_sweep_count(G, O, tol, max_iter):
    """m = 0: the reference's loop still counts its empty sweeps (residual 0:
    one when tol > 0, max_iter when tol = 0), for pull, push and the
    no-allocation entry alike."""
    rp, col, od = np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)
    _, ref_it, ref_hist = O.pr_plain_f32(rp, col, od, tol=tol, max_iter=max_iter)
    with G.Graph(rp, col, od, push=True) as g:
        s, st = g.pagerank(tol=tol, max_iter=max_iter)
        assert s.size == 0 and st.iterations == ref_it and st.residual == 0.0
        assert np.array_equal(g.residuals(), ref_hist)
        _, st = g.pagerank_push(tol=tol, max_iter=max_iter)
        assert st.iterations == ref_it
    import torch
    d = [torch.zeros(n, dtype=t, device="cuda") for n, t in ((1, torch.int32), (0, torch.int32),
                                                             (0, torch.int32), (0, torch.float32))]
    st = G.pagerank_noalloc(0, 0, *d, tol=tol, max_iter=max_iter)
    assert st.iterations == ref_it


def test_edge_cases(G, O):
    # one vertex, no edges
    s, st, _, _ = solve(G, np.array([0, 0], np.int32), np.array([], np.int32),
                        np.array([0], np.int32), tol=1e-3, max_iter=30)
    ref, ref_it, _ = O.pr_plain_f32(np.array([0, 0]), np.array([], np.int32), np.array([0]))
    assert st.iterations == ref_it and np.array_equal(s, ref)
    # no edges at all
    m = 1000
    rp = np.zeros(m + 1, np.int32)
    s, st, _, _ = solve(G, rp, np.array([], np.int32), np.zeros(m, np.int32))
    ref, ref_it, _ = O.pr_plain_f32(rp, np.array([], np.int32), np.zeros(m, np.int32))
    assert st.iterations == ref_it and np.array_equal(s, ref)
    # max_iter = 0 leaves the scores alone
    rp, col, od = erdos_renyi(100, 3, seed=1)
    s, st, _, _ = solve(G, rp, col, od, max_iter=0)
    assert st.iterations == 0 and np.all(s == np.float32(1.0) / np.float32(100))


def test_malformed_csr_rejected(G):
    bad_rp = np.array([0, 2, 1, 3], np.int32)  # not monotone
    with pytest.raises(G.GprError) as e:
        G.Graph(bad_rp, np.array([0, 1, 2], np.int32), np.ones(3, np.int32))
    assert e.value.status == G.GPR_EINVAL
    # columns out of range, from host arrays (checked by the layout build
    # once their copy has landed) and from device arrays (checked up front)
    import torch
    rp, od = np.array([0, 1, 2, 3], np.int32), np.ones(3, np.int32)
    for bad in ([0, 7, 1], [0, -1, 1]):
        col = np.array(bad, np.int32)
        for arrays in ((rp, col, od), tuple(torch.from_numpy(a).cuda() for a in (rp, col, od))):
            with pytest.raises(G.GprError) as e:
                G.Graph(*arrays)
            assert e.value.status == G.GPR_EINVAL
            assert "flags 0x8:" in str(e.value)
    with G.Graph(*(torch.from_numpy(a).cuda() for a in (rp, np.array([0, 2, 1], np.int32), od))):
        pass  # the same arrays with valid columns build


def test_barrier_wait_is_bounded(G, O):
    """A barrier that one CTA too many is expected at never opens: the bounded
    wait must give up, report ETIMEOUT, and leave the graph usable."""
    rp, col, od = O.rmat_graph(10, 8, seed=1)
    with G.Graph(rp, col, od) as g:
        o = G.options(tol=1e-6, max_iter=10, loop=G.LOOP_PERSISTENT, timeout_s=0.05)
        o.reserved[0] = 1
        with pytest.raises(G.GprError) as e:
            g.pagerank(opts=o)
        assert e.value.status == G.GPR_ETIMEOUT
        s, st = g.pagerank(tol=1e-6, max_iter=10)
        ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=10)
        assert np.abs(s - ref).max() <= ABS_TOL


def test_residual_bound_f64(G, O):
    rp, col, od = O.rmat_graph(13, 16, seed=8)
    with G.Graph(rp, col, od) as g:
        s, _ = g.pagerank(tol=1e-6, max_iter=100)
        r = g.residual_f64(s)
    r_ref = O.pr_residual_f64(rp, col, od, s)
    assert abs(r - r_ref) <= 1e-9 * max(1.0, r_ref) + 1e-15


def test_reference_shaped_calls(G, O):
    rp, col, od = O.rmat_graph(11, 16, seed=6)
    m = len(rp) - 1
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od)
    s = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    st = G.PRSolver(m, len(col), rp, col, rp, col, od, s)
    assert abs(st.iterations - ref_it) <= 1 and np.abs(s - ref).max() <= ABS_TOL
    s2 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    G.PageRank(m, len(col), rp, col, od, s2)
    assert np.array_equal(s, s2)


@pytest.mark.parametrize("loop", ["persistent", "graph"])
def test_bf16_mixed_form_matches_plain_accuracy(G, O, loop):
    """Mixed form: BF16 contributions until the change is below 1e-3, then
    FP32 refinement sweeps to the tolerance.  Its FP64-oracle error must match
    the plain FP32 path's (within 10% + 1e-8)."""
    rp, col, od = O.rmat_graph(14, 16, seed=12)
    s64, _, _ = O.pr_f64(rp, col, od)
    lp = G.LOOP_PERSISTENT if loop == "persistent" else G.LOOP_GRAPH
    with G.Graph(rp, col, od) as g:
        plain, sp = g.pagerank(tol=1e-6, max_iter=100, loop=lp)
        mixed, sm = g.pagerank(tol=1e-6, max_iter=100, loop=lp, precision=G.PREC_BF16)
    mx_p, l1_p = O.err_vs_f64(plain, s64)
    mx_m, l1_m = O.err_vs_f64(mixed, s64)
    assert sm.refine_iterations > 0 and sm.iterations > sm.refine_iterations
    assert sm.residual < 1e-6
    assert l1_m <= 1.1 * l1_p + 1e-8 and mx_m <= 1.1 * mx_p + 1e-9


def test_graph_loop_caps_and_reuse(G, O):
    # The CUDA-graph sweep loop (a while node over the per-sweep kernel) stops
    # at max_iter and at tol, matches the persistent loop, and is rebuilt when
    # the options change.
    rp, col, od = O.rmat_graph(13, 8, seed=11)
    with G.Graph(rp, col, od) as g:
        for tol, mi in ((0.0, 7), (1e-6, 60), (0.0, 1), (1e-6, 60), (1e-3, 60)):
            a, sa = g.pagerank(tol=tol, max_iter=mi, loop=G.LOOP_PERSISTENT)
            b, sb = g.pagerank(tol=tol, max_iter=mi, loop=G.LOOP_GRAPH)
            assert sa.iterations == sb.iterations
            assert np.array_equal(a, b)
            assert sb.gpu_launches == 2 + sb.iterations
            if tol == 0.0:
                assert sb.iterations == mi
            ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=tol, max_iter=mi)
            assert abs(sb.iterations - ref_it) <= 1


def test_fp16_form_is_reported_unsupported(G, O):
    """GPR_PREC_FP16 is reserved: each PageRank solver refuses it with
    GPR_EUNSUPPORTED (and the handle stays usable)."""
    rp, col, od = O.rmat_graph(8, 4, seed=1)
    with G.Graph(rp, col, od, batched=True) as g:
        with pytest.raises(G.GprError) as e:
            g.pagerank(precision=G.PREC_FP16)
        assert e.value.status == G.GPR_EUNSUPPORTED
        with pytest.raises(G.GprError) as e:
            g.ppr(np.array([0, 1], np.int32), precision=G.PREC_FP16)
        assert e.value.status == G.GPR_EUNSUPPORTED
        s, st = g.pagerank(tol=1e-4)
        assert st.iterations > 0
    voff = np.array([0, len(rp) - 1], np.int32)
    with G.MultiGraph(rp, col, od, voff) as mg:
        with pytest.raises(G.GprError) as e:
            mg.pagerank(precision=G.PREC_FP16)
        assert e.value.status == G.GPR_EUNSUPPORTED
