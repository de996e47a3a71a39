"""The blocked form of the multi-graph batch (GPR_LAYOUT_BLOCKED on
gpr_multigraph_create, GPR_FORM_BLOCKED on gpr_multigraph_pagerank).

Every graph's rows with in-edges are cut into blocks that never span two
graphs; each block's edges are summed in 64-bit fixed point with one exponent
S for the whole batch (from its edge count and the largest m_g x |initial
score|).  Each graph keeps its own base (1 - d) / m_g, its own FP64 residual
and its own stop rule, as in the units form.  So every sweep of every graph
is pinned exactly by a numpy restatement of the fixed-point recurrence, the
result does not depend on how rows are cut into blocks and tiles, and against
the reference's OpenMP solver (oracle) each graph meets the parity bar:
1e-6 per vertex, sweep count within one.
"""
import math

import numpy as np
import pytest

from graphs import erdos_renyi, zoo
from test_multi_gpu import concat, local

pytestmark = pytest.mark.gpu

KD = np.float32(0.85)


def batch_shift(voff, nnz, s0):
    """The batch's fixed-point exponent (gpr_multi.cu, solve_phase)."""
    sizes = np.diff(voff)
    b0 = max(1.0, float(sizes.max()) * float(np.abs(s0).max()))
    cap = 62 - math.ceil(math.log2(b0))
    pref = math.floor(math.log2(max(1.0, float(nnz)) / b0)) + 28
    return min(cap, max(31, pref))


def fixed_point_sweeps(rp, col, od, s0, sweeps, S):
    """One graph's sweeps with every row summed in 64-bit fixed point 2^-S."""
    m = len(rp) - 1
    base = np.float32(np.float32(1) - KD) / np.float32(m)
    rows = np.repeat(np.arange(m), np.diff(rp))
    s = s0.astype(np.float32).copy()
    for _ in range(sweeps):
        with np.errstate(divide="ignore", invalid="ignore"):
            c = (s / od.astype(np.float32)).astype(np.float32)
        q = np.rint(c[col].astype(np.float64) * 2.0 ** S).astype(np.int64)
        x = np.zeros(m, dtype=np.int64)
        np.add.at(x, rows, q)
        total = (x.astype(np.float64) * 2.0 ** -S).astype(np.float32)
        s = (base + (KD * total).astype(np.float32)).astype(np.float32)
    return s


@pytest.fixture(scope="module")
def batch(O):
    # 12 graphs, sizes log-uniform in [200, 30000]; Chung-Lu ones with hubs
    return O.multigraph(12, 200, 30000, seed=4)


@pytest.mark.parametrize("layout", [{}, {"block_rows": 300, "tile_words": 1024}])
def test_every_sweep_is_the_fixed_point_recurrence(G, O, batch, layout):
    rp, col, od, voff = batch
    n = len(voff) - 1
    with G.MultiGraph(rp, col, od, voff, blocked=True, **layout) as mg:
        s0 = mg.initial_scores()
        S = batch_shift(voff, len(col), s0)
        for sweeps in (1, 3):
            s, iters, _, _ = mg.pagerank(s0.copy(), tol=0.0, max_iter=sweeps, form=G.FORM_BLOCKED)
            assert list(iters) == [sweeps] * n
            for g in range(n):
                a, b = voff[g], voff[g + 1]
                lrp, lcol, lod = local(rp, col, od, voff, g)
                ref = fixed_point_sweeps(lrp, lcol, lod, s0[a:b], sweeps, S)
                assert np.array_equal(s[a:b], ref), (g, sweeps, np.abs(s[a:b] - ref).max())


def test_any_tiling_gives_the_same_bits(G, O, batch):
    rp, col, od, voff = batch
    out = []
    for layout in ({}, {"block_rows": 64, "tile_words": 512}, {"block_rows": 1000,
                                                                "tile_words": 2048},
                   {"block_rows": 12288, "tile_words": 4096}):
        with G.MultiGraph(rp, col, od, voff, blocked=True, **layout) as mg:
            s, iters, res, _ = mg.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
        out.append((s, iters, res))
    # (the residuals are sums of per-tile partial sums, so their last bits
    # follow the tiling; the scores do not)
    for s, iters, res in out[1:]:
        assert np.array_equal(s, out[0][0]) and np.array_equal(iters, out[0][1])
        assert np.allclose(res, out[0][2], rtol=1e-12, atol=0)


@pytest.mark.parametrize("tol", [1e-6, 1e-4])
def test_blocked_batch_matches_reference(G, O, batch, tol):
    rp, col, od, voff = batch
    n = len(voff) - 1
    with G.MultiGraph(rp, col, od, voff, blocked=True) as mg:
        s, iters, _, st = mg.pagerank(tol=tol, max_iter=100, form=G.FORM_BLOCKED)
        units, it_u, _, _ = mg.pagerank(tol=tol, max_iter=100, form=G.FORM_EXACT)
    for g in range(n):
        a, b = voff[g], voff[g + 1]
        lrp, lcol, lod = local(rp, col, od, voff, g)
        ref, ref_it, _ = O.pr_plain_f32(lrp, lcol, lod, tol=tol, max_iter=100)
        assert abs(int(iters[g]) - ref_it) <= 1, g
        assert abs(int(iters[g]) - int(it_u[g])) <= 1, g
        s64, _, _ = O.pr_f64(lrp, lcol, lod, tol=0.0, max_iter=int(iters[g]))
        assert np.all(np.abs(s[a:b] - ref) <= 1e-6 + np.abs(ref - s64)), g


def test_edge_cases(G, O):
    # empty graph, one vertex, edge-free graph, a normal graph, a star hub
    empty = (np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    one = (np.zeros(2, np.int32), np.zeros(0, np.int32), np.zeros(1, np.int32))
    bare = (np.zeros(301, np.int32), np.zeros(0, np.int32), np.zeros(300, np.int32))
    er = erdos_renyi(5000, 6, seed=9)
    m = 9000
    hub_rp = np.array([0, m - 1] + [m - 1] * (m - 1), np.int32)
    hub = (hub_rp, np.arange(1, m).astype(np.int32),
           np.concatenate([[0], np.ones(m - 1)]).astype(np.int32))
    parts = [empty, one, er, bare, hub, empty]
    rp, col, od, voff = concat(parts)
    for tol, mi in ((1e-6, 50), (0.0, 7), (1e-6, 0)):
        with G.MultiGraph(rp, col, od, voff, blocked=True, block_rows=700) as mg:
            s, iters, res, _ = mg.pagerank(tol=tol, max_iter=mi, form=G.FORM_BLOCKED)
        for g, (lrp, lcol, lod) in enumerate(parts):
            a, b = voff[g], voff[g + 1]
            with np.errstate(divide="ignore"):
                ref, ref_it, _ = O.pr_plain_f32(lrp, lcol, lod, tol=tol, max_iter=mi)
            assert abs(int(iters[g]) - ref_it) <= 1 if b > a else iters[g] == ref_it, (g, tol, mi)
            if b == a:
                assert res[g] == 0.0
                continue
            s64, _, _ = O.pr_f64(lrp, lcol, lod, tol=0.0, max_iter=int(iters[g]))
            assert np.all(np.abs(s[a:b] - ref) <= 1e-6 + np.abs(ref - s64)), (g, tol, mi)


def test_forms_and_errors(G, O, batch):
    rp, col, od, voff = batch
    with G.MultiGraph(rp, col, od, voff) as mg:
        with pytest.raises(G.GprError) as e:
            mg.pagerank(tol=1e-6, max_iter=50, form=G.FORM_BLOCKED)
        assert e.value.status == G.GPR_EINVAL
        exact, it_e, _, _ = mg.pagerank(tol=1e-6, max_iter=50)
    with G.MultiGraph(rp, col, od, voff, blocked=True) as mg:
        # AUTO below 50.3M edges, and the graph loop: the units form
        auto, it_a, _, _ = mg.pagerank(tol=1e-6, max_iter=50)
        assert np.array_equal(auto, exact) and np.array_equal(it_a, it_e)
        looped, _, _, _ = mg.pagerank(tol=1e-6, max_iter=50, loop=G.LOOP_GRAPH)
        assert np.array_equal(looped, exact)
        for kw in ({"loop": G.LOOP_GRAPH}, {"precision": G.PREC_BF16}):
            with pytest.raises(G.GprError) as e:
                mg.pagerank(tol=1e-6, max_iter=50, form=G.FORM_BLOCKED, **kw)
            assert e.value.status == G.GPR_EUNSUPPORTED
        with pytest.raises(G.GprError) as e:
            mg.pagerank(tol=1e-6, max_iter=50, form=9)
        assert e.value.status == G.GPR_EINVAL
        # a non-finite score: refused by the blocked form
        bad = mg.initial_scores()
        bad[3] = np.inf
        with pytest.raises(G.GprError) as e:
            mg.pagerank(bad.copy(), tol=1e-6, max_iter=5, form=G.FORM_BLOCKED)
        assert e.value.status == G.GPR_EINVAL
        # the handle stays usable
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=50, form=G.FORM_BLOCKED)
        assert np.all(np.abs(s - exact) <= 1e-6)


def test_blocked_barrier_wait_is_bounded(G, O, batch):
    rp, col, od, voff = batch
    with G.MultiGraph(rp, col, od, voff, blocked=True) as mg:
        o = G.options(tol=1e-6, max_iter=20, timeout_s=0.05, form=G.FORM_BLOCKED)
        o.reserved[0] = 1
        with pytest.raises(G.GprError) as e:
            mg.pagerank(opts=o)
        assert e.value.status == G.GPR_ETIMEOUT
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=20, form=G.FORM_BLOCKED)
        s2, iters2, _, _ = mg.pagerank(tol=1e-6, max_iter=20, form=G.FORM_BLOCKED)
    assert np.array_equal(s, s2) and np.array_equal(iters, iters2)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_zoo_batch_is_the_fixed_point_recurrence(G, O, seed):
    """A batch of random shapes (and an empty graph) cut into random blocks:
    three sweeps of every graph bit for bit the fixed-point restatement."""
    rng = np.random.default_rng(seed)
    kinds = ["er", "power", "chain", "islands", "sink"]
    parts = [zoo(kinds[i % 5], 10 * seed + i) for i in range(int(rng.integers(3, 9)))]
    parts.insert(int(rng.integers(0, len(parts))),
                 (np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)))
    rp, col, od, voff = concat(parts)
    layout = dict(block_rows=int(rng.integers(1, 12289)), tile_words=int(rng.integers(512, 1 << 17)))
    with G.MultiGraph(rp, col, od, voff, blocked=True, **layout) as mg:
        s0 = mg.initial_scores()
        S = batch_shift(voff, len(col), s0)
        s, iters, _, _ = mg.pagerank(s0.copy(), tol=0.0, max_iter=3, form=G.FORM_BLOCKED)
    for g, (lrp, lcol, lod) in enumerate(parts):
        a, b = voff[g], voff[g + 1]
        if b == a:
            continue
        assert iters[g] == 3
        ref = fixed_point_sweeps(lrp, lcol, lod, s0[a:b], 3, S)
        assert np.array_equal(s[a:b], ref), (seed, g, layout)
