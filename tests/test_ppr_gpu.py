"""Batched personalized PageRank on the GPU against the FP64 oracle.

The reference has no personalized PageRank; oracle/oracle.c orc_ppr_f64
defines the semantics (teleport mass and dangling mass returned to the
seed, per-vector stop at L1 change < tol).  Bars: FP32 form, every vector's
L1 error vs the FP64 oracle <= 1e-5 and its sweep count within one.  BF16
form: BF16 contributions until the change drops below 1e-3, then FP32
refinement sweeps to the same tolerance -- the same L1 bar, 1e-5.
"""
import numpy as np
import pytest

from graphs import star

pytestmark = pytest.mark.gpu


def l1_per_vector(x, ref):
    return np.abs(x.astype(np.float64) - ref).sum(axis=0)


@pytest.mark.parametrize("k", [1, 5, 8, 16, 32, 40, 64, 128])
def test_ppr_fp32_matches_fp64_oracle(G, O, k):
    rp, col, od = O.rmat_graph(12, 8, seed=31)
    m = len(rp) - 1
    seeds = O.uniform_int(k, 77, m)
    ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od, batched=True) as g:
        x, it, st = g.ppr(seeds, tol=1e-6, max_iter=100)
    assert np.all(l1_per_vector(x, ref) <= 1e-5)
    assert np.all(np.abs(it - ref_it) <= 1)
    np.testing.assert_allclose(x.sum(axis=0), ref.sum(axis=0), atol=1e-5)


def test_ppr_bf16_form(G, O):
    """BF16 contributions to a change below 1e-3, then FP32 refinement until
    the change is below tol (1-d)/d: the BF16 start leaves its error in the
    slowest modes, and that stop bounds what is left of it by tol, so the
    result is about as close to the FP64 fixed point as the FP32 form's."""
    rp, col, od = O.rmat_graph(12, 8, seed=32)
    m = len(rp) - 1
    seeds = O.uniform_int(32, 78, m)
    fixed, _ = O.ppr_f64(rp, col, od, seeds, tol=1e-15, max_iter=3000)
    with G.Graph(rp, col, od, batched=True) as g:
        x, it, st = g.ppr(seeds, tol=1e-6, max_iter=200, precision=G.PREC_BF16)
        x32, it32, _ = g.ppr(seeds, tol=1e-6, max_iter=200)
    assert st.refine_iterations > 0
    e16, e32 = l1_per_vector(x, fixed), l1_per_vector(x32, fixed)
    assert np.all(e16 <= 1e-5)
    assert e16.max() <= 2 * e32.max() + 1.5e-6
    assert np.all(it <= it32 + 60)


def test_ppr_seed_without_in_edges_and_chunked_hub(G, O):
    rp, col, od = star(60000)
    m = len(rp) - 1
    indeg = np.diff(rp)
    zero_in = int(np.flatnonzero(indeg == 0)[0])
    seeds = np.array([0, 1, zero_in, zero_in, 12345], dtype=np.int32)
    ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od, batched=True, chunk=512, chunk_min=1024) as g:
        lay = g.layout()
        x, it, st = g.ppr(seeds, tol=1e-6, max_iter=100)
    assert lay["n_chunks"] > lay["n_long"] > 0
    assert np.all(l1_per_vector(x, ref) <= 1e-5)
    assert np.all(np.abs(it - ref_it) <= 1)


def test_ppr_requires_batched_layout(G, O):
    rp, col, od = O.rmat_graph(8, 4, seed=1)
    with G.Graph(rp, col, od) as g:
        with pytest.raises(G.GprError) as e:
            g.ppr(np.array([0], np.int32))
    assert e.value.status == G.GPR_EINVAL


@pytest.mark.parametrize("k,prec", [(8, "fp32"), (32, "fp32"), (128, "fp32"), (32, "bf16")])
def test_ppr_graph_loop_matches_persistent(G, O, k, prec):
    """GPR_LOOP_GRAPH runs one sweep per launch inside a CUDA-graph while
    loop (the last CTA to finish a sweep closes it).  The sweep code and the
    CTA-order reductions are the persistent kernel's, so scores and sweep
    counts are bit-identical."""
    rp, col, od = O.rmat_graph(12, 8, seed=33)
    seeds = O.uniform_int(k, 79, len(rp) - 1)
    p = G.PREC_BF16 if prec == "bf16" else G.PREC_FP32
    with G.Graph(rp, col, od, batched=True) as g:
        x0, it0, st0 = g.ppr(seeds, tol=1e-6, max_iter=100, precision=p, loop=G.LOOP_PERSISTENT)
        x1, it1, st1 = g.ppr(seeds, tol=1e-6, max_iter=100, precision=p, loop=G.LOOP_GRAPH)
    np.testing.assert_array_equal(x0, x1)
    np.testing.assert_array_equal(it0, it1)
    assert st1.iterations == st0.iterations
    assert st1.refine_iterations == st0.refine_iterations
    # one launch per sweep plus the launch that finds the phase done
    assert st1.gpu_launches > st0.gpu_launches


def test_ppr_graph_loop_hub_chunks_and_cap(G, O):
    """A hub of 60,000 in-edges (many chunks summed by the last arriving warp)
    in graph mode, and the max_iter cap of the graph loop."""
    rp, col, od = star(60000)
    seeds = np.array([0, 1, 12345], dtype=np.int32)
    ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od, batched=True) as g:
        x, it, st = g.ppr(seeds, tol=1e-6, max_iter=100, loop=G.LOOP_GRAPH)
        xc, itc, stc = g.ppr(seeds, tol=0.0, max_iter=4, loop=G.LOOP_GRAPH)
        xp, itp, stp = g.ppr(seeds, tol=0.0, max_iter=4)
    assert np.all(l1_per_vector(x, ref) <= 1e-5)
    assert np.all(np.abs(it - ref_it) <= 1)
    assert stc.iterations == 4 and np.all(itc == 4)
    np.testing.assert_array_equal(xc, xp)


@pytest.mark.parametrize("loop", ["persistent", "graph"])
def test_ppr_graphs_without_edges(G, O, loop):
    """No row has an in-edge: no work units, an empty packet table; every
    seed keeps its mass (x = e_seed after one sweep), as in the oracle."""
    lp = G.LOOP_GRAPH if loop == "graph" else G.LOOP_PERSISTENT
    col = np.zeros(0, np.int32)
    for m, seeds in ((5, [0, 3, 3]), (1, [0])):
        rp, od = np.zeros(m + 1, np.int32), np.zeros(m, np.int32)
        seeds = np.array(seeds, np.int32)
        ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
        with G.Graph(rp, col, od, batched=True) as g:
            x, it, st = g.ppr(seeds, tol=1e-6, max_iter=100, loop=lp)
        np.testing.assert_array_equal(x, ref.astype(np.float32))
        np.testing.assert_array_equal(it, ref_it)


def test_ppr_barrier_wait_is_bounded(G, O):
    """A grid barrier that expects one CTA too many never opens: every wait
    gives up after timeout_s, the solve reports ETIMEOUT, and the graph
    still solves correctly afterwards (no GPU fault, no hang)."""
    rp, col, od = O.rmat_graph(10, 8, seed=1)
    seeds = O.uniform_int(8, 5, len(rp) - 1)
    with G.Graph(rp, col, od, batched=True) as g:
        o = G.options(tol=1e-6, max_iter=10, loop=G.LOOP_PERSISTENT, timeout_s=0.05)
        o.reserved[0] = 1
        with pytest.raises(G.GprError) as e:
            g.ppr(seeds, opts=o)
        assert e.value.status == G.GPR_ETIMEOUT
        x, it, st = g.ppr(seeds, tol=1e-6, max_iter=100)
    ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    assert np.all(l1_per_vector(x, ref) <= 1e-5)
    assert np.all(np.abs(it - ref_it) <= 1)


def mixed_seeds(O, rp, od, k, seed):
    """k seeds, about half on vertices without out-edges (their vector keeps
    its mass at the seed and stops after one sweep), the rest on vertices with
    in- and out-edges: the active set halves after the first sweep."""
    rng = np.random.default_rng(seed)
    dang = np.flatnonzero(od == 0)
    live = np.flatnonzero((np.diff(rp) > 0) & (od > 0))
    n_dead = k // 2 + 1 if k >= 16 else 0
    return np.concatenate([rng.choice(dang, n_dead), rng.choice(live, k - n_dead)]).astype(np.int32)


@pytest.mark.parametrize("k", [16, 32, 128])
@pytest.mark.parametrize("loop", ["persistent", "graph"])
def test_ppr_packing_matches_unpacked(G, O, k, loop):
    """Once at most half of the vectors are still updating, the solve goes on
    with those packed into the next narrower layout (gpr_pr_opts.ppr_repack,
    on by default).  The narrower layout sums each row in another order, so
    against the unpacked solve the results agree within rounding (1e-6 per
    entry, sweeps within one); both meet the FP64 oracle's bar."""
    lp = G.LOOP_GRAPH if loop == "graph" else G.LOOP_PERSISTENT
    rp, col, od = O.rmat_graph(13, 8, seed=41)
    seeds = mixed_seeds(O, rp, od, k, 5)
    ref, ref_it = O.ppr_f64(rp, col, od, seeds, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od, batched=True) as g:
        xa, ita, sta = g.ppr(seeds, tol=1e-6, max_iter=100, loop=lp)
        xb, itb, stb = g.ppr(seeds, tol=1e-6, max_iter=100, loop=lp, ppr_repack=False)
        xc, itc, stc = g.ppr(seeds, tol=1e-6, max_iter=100, loop=lp)
    for x, it in ((xa, ita), (xb, itb)):
        assert np.all(l1_per_vector(x, ref) <= 1e-5)
        assert np.all(np.abs(it - ref_it) <= 1)
    assert np.all(np.abs(ita - itb) <= 1)
    assert np.abs(xa - xb).max() <= 1e-6
    # packing launched its pack / unpack kernels; repeated solves are identical
    assert sta.gpu_launches > stb.gpu_launches
    np.testing.assert_array_equal(xa, xc)
    np.testing.assert_array_equal(ita, itc)


def test_ppr_packing_in_the_bf16_refinement(G, O):
    rp, col, od = O.rmat_graph(12, 8, seed=42)
    seeds = mixed_seeds(O, rp, od, 32, 6)
    fixed, _ = O.ppr_f64(rp, col, od, seeds, tol=1e-15, max_iter=3000)
    with G.Graph(rp, col, od, batched=True) as g:
        xa, ita, sta = g.ppr(seeds, tol=1e-6, max_iter=200, precision=G.PREC_BF16)
        xb, itb, stb = g.ppr(seeds, tol=1e-6, max_iter=200, precision=G.PREC_BF16,
                             ppr_repack=False)
    assert sta.refine_iterations > 0
    assert np.all(l1_per_vector(xa, fixed) <= 1e-5)
    assert np.abs(xa - xb).max() <= 1e-6 and np.all(np.abs(ita - itb) <= 1)


def test_ppr_packing_with_a_sweep_cap(G, O):
    """The sweep budget is shared by the layouts: a capped solve stops at
    max_iter sweeps in total, as the unpacked one does."""
    rp, col, od = O.rmat_graph(12, 8, seed=43)
    seeds = mixed_seeds(O, rp, od, 32, 7)
    with G.Graph(rp, col, od, batched=True) as g:
        xa, ita, sta = g.ppr(seeds, tol=1e-9, max_iter=9)
        xb, itb, stb = g.ppr(seeds, tol=1e-9, max_iter=9, ppr_repack=False)
    assert sta.iterations == stb.iterations == 9
    np.testing.assert_array_equal(ita, itb)
    assert np.abs(xa - xb).max() <= 1e-6
