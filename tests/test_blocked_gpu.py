"""The blocked form of the PageRank sweep (GPR_LAYOUT_BLOCKED, GPR_FORM_BLOCKED).

Rows are summed block by block from source-ordered edges in 64-bit fixed
point, except rows with more than chunk_min in-edges that either exceed
blocked_long or (blocked_long 0, the default) would hold more than 1/8 of the
edges of their block: each contribution c (FP32) becomes
rint(c * 2^S), the row's integers are added exactly, and the sum is
(float)(x * 2^-S).  The update is the reference's (src/pr/omp_base.cc:39, 26).
So the form is pinned exactly: on graphs without chunked rows every sweep is
restated here in numpy and compared bit for bit, and the result does not
depend on how the rows are cut into blocks and tiles.  Against the reference's
OpenMP solver (oracle) it meets the parity bar of the other forms: 1e-6 per
vertex, sweep count within one.
"""
import math

import numpy as np
import pytest

from graphs import degree_ladder, erdos_renyi, star, zoo

pytestmark = pytest.mark.gpu

ABS_TOL = 1e-6
KD = np.float32(0.85)


def shift(m, nnz, mx):
    """The fixed-point exponent the library picks (gpr_pagerank.cu, blocked_shift)."""
    b0 = max(1.0, float(m) * float(mx))
    cap = 62 - math.ceil(math.log2(b0))
    pref = math.floor(math.log2(max(1.0, float(nnz)) / b0)) + 28
    return min(cap, max(31, pref))


def fixed_point_sweeps(rp, col, od, s0, sweeps):
    """The blocked form restated: every row summed in 64-bit fixed point."""
    m = len(rp) - 1
    S = shift(m, len(col), np.abs(s0).max())
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
    return s, S


def solve(G, rp, col, od, layout=None, **kw):
    with G.Graph(rp, col, od, blocked=True, **(layout or {})) as g:
        s, st = g.pagerank(**kw)
        return s, st


@pytest.mark.parametrize("maker", ["er", "rmat"])
def test_every_sweep_is_the_fixed_point_recurrence(G, O, maker):
    if maker == "er":
        rp, col, od = erdos_renyi(40000, 8, seed=11)
    else:
        rp, col, od = O.rmat_graph(13, 8, seed=2)
    assert np.diff(rp).max() <= 4096  # no chunked rows: every row is blocked
    m = len(rp) - 1
    s0 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    for sweeps in (1, 2, 7):
        s, st = solve(G, rp, col, od, tol=0.0, max_iter=sweeps, form=G.FORM_BLOCKED)
        assert st.iterations == sweeps
        ref, S = fixed_point_sweeps(rp, col, od, s0, sweeps)
        assert S >= 31
        assert np.array_equal(s, ref), (sweeps, np.abs(s - ref).max())


def test_any_tiling_gives_the_same_bits(G, O):
    rp, col, od = O.rmat_graph(14, 16, seed=4)
    ref, st_ref = solve(G, rp, col, od, tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
    for block_rows, tile_words in ((64, 512), (1000, 2048), (7, 512), (12288, 4096)):
        s, st = solve(G, rp, col, od, dict(block_rows=block_rows, tile_words=tile_words),
                      tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
        assert st.iterations == st_ref.iterations
        assert np.array_equal(s, ref), (block_rows, tile_words)
    again, _ = solve(G, rp, col, od, tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
    assert np.array_equal(again, ref)


@pytest.mark.parametrize("scale,tol", [(16, 1e-4), (15, 1e-6)])
def test_blocked_matches_reference(G, O, scale, tol):
    rp, col, od = O.rmat_graph(scale, 16, seed=1)
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=tol, max_iter=100)
    s, st = solve(G, rp, col, od, tol=tol, max_iter=100, form=G.FORM_BLOCKED)
    assert abs(st.iterations - ref_it) <= 1
    assert np.abs(s - ref).max() <= ABS_TOL
    # Rounding: against an FP64 run of the same sweeps, the fixed-point sums
    # are at least as close as the reference's float sums.
    n = st.iterations
    ref_n = ref if n == ref_it else O.pr_plain_f32(rp, col, od, tol=0.0, max_iter=n)[0]
    s64n, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=n)
    mx_g, l1_g = O.err_vs_f64(s, s64n)
    mx_r, l1_r = O.err_vs_f64(ref_n, s64n)
    assert l1_g <= l1_r and mx_g <= mx_r
    # Both are reported against the FP64 fixed point; there the stopping
    # point, not the summation, dominates.
    s64, _, _ = O.pr_f64(rp, col, od)
    _, l1_fix = O.err_vs_f64(s, s64)
    assert l1_fix <= 1e-5 if tol <= 1e-6 else True


@pytest.mark.parametrize("maker", [lambda: star(20000), degree_ladder], ids=["star", "ladder"])
def test_heavy_rows_in_blocks_follow_the_fixed_point_recurrence(G, O, maker):
    """Rows the exact-order layout cuts into chunks (chunk_min 1024) are summed
    in blocks when they have at most blocked_long in-edges: every sweep is
    still the fixed-point recurrence, bit for bit, hub rows included (a hub
    that crowds its block only costs time)."""
    rp, col, od = maker()
    m = len(rp) - 1
    assert np.diff(rp).max() > 1024
    s0 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    for layout in (dict(block_rows=300, tile_words=1024), {}):
        with G.Graph(rp, col, od, chunk=512, chunk_min=1024, blocked=True,
                     blocked_long=1 << 30, **layout) as g:
            assert g.layout()["n_long"] > 0
            for sweeps in (1, 3):
                s, st = g.pagerank(tol=0.0, max_iter=sweeps, form=G.FORM_BLOCKED)
                ref, _ = fixed_point_sweeps(rp, col, od, s0, sweeps)
                assert np.array_equal(s, ref), (layout, sweeps, np.abs(s - ref).max())


@pytest.mark.parametrize("maker", [lambda: star(20000), degree_ladder], ids=["star", "ladder"])
@pytest.mark.parametrize("blocked_long", [0, 64, 2048, 4096, 1 << 30])
def test_heavy_row_threshold(G, O, maker, blocked_long):
    """Rows above blocked_long in-edges (0: the rows that crowd their block)
    are summed in chunks, the rest in blocks; any split meets the parity bar."""
    rp, col, od = maker()
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od, chunk=256, chunk_min=64, blocked=True, block_rows=500,
                 tile_words=2048, blocked_long=blocked_long) as g:
        s, st = g.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
    assert abs(st.iterations - ref_it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=st.iterations)
    assert np.all(np.abs(s - ref) <= ABS_TOL + np.abs(ref - s64))
    with pytest.raises(G.GprError) as e:
        G.Graph(rp, col, od, blocked=True, blocked_long=-1)
    assert e.value.status == G.GPR_EINVAL


@pytest.mark.parametrize("maker", [star, degree_ladder])
def test_blocked_with_chunked_rows(G, O, maker):
    rp, col, od = maker()
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-5, max_iter=60)
    with G.Graph(rp, col, od, chunk=512, chunk_min=1024, blocked=True, block_rows=300,
                 tile_words=1024, blocked_long=1) as g:
        lay = g.layout()
        s, st = g.pagerank(tol=1e-5, max_iter=60, form=G.FORM_BLOCKED)
    assert lay["n_long"] > 0
    assert abs(st.iterations - ref_it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=st.iterations)
    assert np.all(np.abs(s - ref) <= ABS_TOL + np.abs(ref - s64))


def test_forms_on_one_graph(G, O):
    rp, col, od = O.rmat_graph(12, 16, seed=3)
    with G.Graph(rp, col, od) as g:
        plain, st_p = g.pagerank(tol=1e-6, max_iter=100)
        with pytest.raises(G.GprError) as e:
            g.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
        assert e.value.status == G.GPR_EINVAL
    with G.Graph(rp, col, od, blocked=True) as g:
        exact, st_e = g.pagerank(tol=1e-6, max_iter=100, form=G.FORM_EXACT)
        assert st_e.iterations == st_p.iterations and np.array_equal(exact, plain)
        # the per-sweep graph loop runs the exact-order form
        looped, _ = g.pagerank(tol=1e-6, max_iter=100, loop=G.LOOP_GRAPH)
        assert np.array_equal(looped, plain)
        with pytest.raises(G.GprError) as e:
            g.pagerank(tol=1e-6, max_iter=100, loop=G.LOOP_GRAPH, form=G.FORM_BLOCKED)
        assert e.value.status == G.GPR_EUNSUPPORTED
        with pytest.raises(G.GprError) as e:
            g.pagerank(tol=1e-6, max_iter=100, form=7)
        assert e.value.status == G.GPR_EINVAL
        blocked, st_b = g.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
        assert abs(st_b.iterations - st_p.iterations) <= 1
        assert np.abs(blocked - plain).max() <= ABS_TOL


def test_nonfinite_scores(G, O):
    rp, col, od = O.rmat_graph(10, 8, seed=9)
    m = len(rp) - 1
    s0 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    s0[5] = np.inf
    with G.Graph(rp, col, od) as g:
        ref, st_ref = g.pagerank(s0.copy(), tol=1e-6, max_iter=5)
    with G.Graph(rp, col, od, blocked=True) as g:
        s, st = g.pagerank(s0.copy(), tol=1e-6, max_iter=5)  # AUTO: the exact-order form
        assert st.iterations == st_ref.iterations
        assert np.array_equal(np.isnan(s), np.isnan(ref))
        assert np.array_equal(s[~np.isnan(s)], ref[~np.isnan(ref)])
        with pytest.raises(G.GprError) as e:
            g.pagerank(s0.copy(), tol=1e-6, max_iter=5, form=G.FORM_BLOCKED)
        assert e.value.status == G.GPR_EINVAL


def test_scores_of_any_magnitude(G, O):
    """Initial scores far from 1/m: the exponent shrinks so no row's sum can
    leave the 64-bit range; the sweeps still follow the fixed-point recurrence."""
    rp, col, od = erdos_renyi(5000, 6, seed=2)
    m = len(rp) - 1
    for scale in (1e6, -3.0, 1e-20):
        s0 = (np.random.default_rng(1).random(m).astype(np.float32) * np.float32(scale))
        s, st = solve(G, rp, col, od, scores=s0.copy(), tol=0.0, max_iter=3,
                      form=G.FORM_BLOCKED)
        ref, _ = fixed_point_sweeps(rp, col, od, s0, 3)
        assert np.array_equal(s, ref), scale


def test_graphs_without_blocked_rows(G, O):
    # no edges: only zero-in-degree rows
    rp = np.zeros(101, dtype=np.int32)
    od = np.zeros(100, dtype=np.int32)
    s, st = solve(G, rp, np.zeros(0, dtype=np.int32), od, tol=1e-6, max_iter=10,
                  form=G.FORM_BLOCKED)
    ref, it, _ = O.pr_plain_f32(rp, np.zeros(0, np.int32), od, tol=1e-6, max_iter=10)
    assert st.iterations == it and np.array_equal(s, ref)
    # every row with in-edges chunked
    rp, col, od = star(20000)
    with G.Graph(rp, col, od, chunk=128, chunk_min=1, blocked=True, blocked_long=1) as g:
        s, st = g.pagerank(tol=1e-6, max_iter=50, form=G.FORM_BLOCKED)
    ref, it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=50)
    assert abs(st.iterations - it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=st.iterations)
    assert np.all(np.abs(s - ref) <= ABS_TOL + np.abs(ref - s64))


def test_blocked_barrier_wait_is_bounded(G, O):
    rp, col, od = O.rmat_graph(10, 8, seed=1)
    with G.Graph(rp, col, od, blocked=True) as g:
        o = G.options(tol=1e-6, max_iter=10, timeout_s=0.05, form=G.FORM_BLOCKED)
        o.reserved[0] = 1
        with pytest.raises(G.GprError) as e:
            g.pagerank(opts=o)
        assert e.value.status == G.GPR_ETIMEOUT
        s, st = g.pagerank(tol=1e-6, max_iter=10, form=G.FORM_BLOCKED)
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=10)
    assert np.abs(s - ref).max() <= ABS_TOL


@pytest.mark.parametrize("kind", ["er", "power", "chain", "islands", "sink"])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_graph_zoo_is_the_fixed_point_recurrence(G, O, kind, seed):
    """Random shapes and random cuts into blocks and tiles (one or two CTAs
    per SM): two sweeps bit for bit the fixed-point restatement, and a solve
    to tol 1e-6 within the parity bar of the oracle."""
    rp, col, od = zoo(kind, seed)
    m = len(rp) - 1
    rng = np.random.default_rng(100 * seed + len(kind))
    layout = dict(block_rows=int(rng.integers(1, 12289)), tile_words=int(rng.integers(512, 1 << 17)),
                  blocked_long=1 << 30)
    s0 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    with G.Graph(rp, col, od, blocked=True, **layout) as g:
        s, st = g.pagerank(tol=0.0, max_iter=2, form=G.FORM_BLOCKED)
        ref, _ = fixed_point_sweeps(rp, col, od, s0, 2)
        assert np.array_equal(s, ref), (kind, seed, layout)
        s, st = g.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=100)
    assert abs(st.iterations - ref_it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=st.iterations)
    assert np.all(np.abs(s - ref) <= ABS_TOL + np.abs(ref - s64))
