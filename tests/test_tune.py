"""Autotuner: distribution signatures and the cache (CPU), the search on the
GPU (the pick must solve to the same answer as the defaults)."""
import os

import numpy as np
import pytest

from graphs import erdos_renyi, star

LAYOUT_KEYS = ("sell_max", "chunk", "chunk_min", "hot_entries", "blocked", "block_rows",
               "tile_words", "blocked_long")


def test_signature_classes(G, O):
    rp, _, _ = erdos_renyi(10000, 8, 1)
    assert G.tune_signature(rp) == "pr:m13:d3:s0"
    assert G.tune_signature(rp, batch=True) == "batch:d3:s0"
    rp, _, _ = star(20000)
    assert G.tune_signature(rp).endswith(":s2")  # one vertex holds every edge
    rp, _, _ = O.rmat_graph(12, 16, seed=1)
    assert G.tune_signature(rp).startswith("pr:m12:")


def test_cache_lookup_later_lines_win(G, tmp_path):
    p = str(tmp_path / "tune.txt")
    with open(p, "w") as f:
        f.write("pr:m14:d4:s2 32 4096 4096 16384 3 0.5\n")
        f.write("pr:m14:d4:s2 16 1024 1024 8192 5 0.25\n")
        f.write("batch:d3:s0 128 4096 16384 32768 0 1.5\n")
    r = G.tune_cache_lookup(p, "pr:m14:d4:s2")
    assert r["sell_max"] == 16 and r["chunk_min"] == 1024 and r["variant"] == 5
    assert r["hot_entries"] == 8192 and r["from_cache"] and r["ms_per_sweep"] == 0.25
    assert G.tune_cache_lookup(p, "batch:d3:s0")["sell_max"] == 128
    assert G.tune_cache_lookup(p, "pr:m1:d1:s1") is None
    assert not G.tune_cache_lookup(p, "pr:m14:d4:s2")["blocked"]


def test_cache_entries_of_the_blocked_form(G, tmp_path):
    p = str(tmp_path / "tune.txt")
    with open(p, "w") as f:
        f.write("pr:m24:d4:s2 64 4096 1073741824 32768 0 0.59 4 8192 131072\n")
        f.write("pr:m22:d4:s2 64 4096 4096 32768 0 0.15 4 0 0 16384\n")
    r = G.tune_cache_lookup(p, "pr:m24:d4:s2")
    assert r["blocked"] and r["block_rows"] == 8192 and r["tile_words"] == 131072
    assert r["chunk_min"] == 1 << 30 and r["ms_per_sweep"] == 0.59
    assert r["blocked_long"] == 0  # ten-field lines: the library default
    r = G.tune_cache_lookup(p, "pr:m22:d4:s2")
    assert r["blocked"] and r["blocked_long"] == 16384 and r["block_rows"] == 0


@pytest.mark.gpu
def test_tune_graph_and_cache(G, O, tmp_path):
    rp, col, od = O.rmat_graph(15, 16, seed=2)
    cache = str(tmp_path / "tune.txt")
    r = G.tune_graph(rp, col, od, cache=cache, sweeps=4)
    assert not r["from_cache"] and r["candidates"] >= 8
    assert r["ms_per_sweep"] <= r["default_ms_per_sweep"]  # a pick only replaces a slower one
    assert os.path.exists(cache)
    r2 = G.tune_graph(rp, col, od, cache=cache, sweeps=4)
    assert r2["from_cache"] and r2["signature"] == r["signature"]
    for k in LAYOUT_KEYS + ("variant",):
        assert r2[k] == r[k]
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=100)
    with G.Graph(rp, col, od, **{k: r[k] for k in LAYOUT_KEYS}) as g:
        s, st = g.pagerank(tol=1e-6, max_iter=100, variant=r["variant"])
    assert abs(st.iterations - ref_it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=st.iterations)
    assert np.all(np.abs(s - ref) <= 1e-6 + np.abs(ref - s64))


@pytest.mark.gpu
def test_tune_multigraph(G, O, tmp_path):
    rp, col, od, voff = O.multigraph(10, 300, 20000, seed=6)
    cache = str(tmp_path / "tune.txt")
    lays, r = G.tune_multigraph(rp, col, od, voff, cache=cache, sweeps=4)
    assert len(lays) == 10 and r["signature"].startswith("batch:")
    with G.MultiGraph(rp, col, od, voff, layouts=lays) as mg:
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=100)
    for g in range(10):
        a, b = voff[g], voff[g + 1]
        e0, e1 = rp[a], rp[b]
        lrp, lcol, lod = rp[a:b + 1] - e0, col[e0:e1] - a, od[a:b]
        ref, ref_it, _ = O.pr_plain_f32(lrp, lcol, lod, tol=1e-6, max_iter=100)
        assert abs(int(iters[g]) - ref_it) <= 1
        s64, _, _ = O.pr_f64(lrp, lcol, lod, tol=0.0, max_iter=int(iters[g]))
        assert np.all(np.abs(s[a:b] - ref) <= 1e-6 + np.abs(ref - s64))
    lays2, r2 = G.tune_multigraph(rp, col, od, voff, cache=cache, sweeps=4)
    assert lays2 == lays and r2["candidates"] == 1


@pytest.mark.gpu
def test_tune_multigraph_blocked_pick_reaches_the_batch(G, O, tmp_path):
    """A blocked pick (here written into the cache, as the tuner writes it
    when the blocked form wins) comes back in every graph's layout and builds
    the batch's blocked form, which then solves like the units form."""
    rp, col, od, voff = O.multigraph(10, 300, 20000, seed=6)
    cache = str(tmp_path / "tune.txt")
    sigs = {G.tune_signature(rp[voff[g]:voff[g + 1] + 1] - rp[voff[g]], batch=True)
            for g in range(10)}
    with open(cache, "w") as f:
        for s in sorted(sigs):  # flags 4: GPR_LAYOUT_BLOCKED
            f.write(f"{s} 64 4096 4096 32768 0 0.5 4 300 1024 0\n")
    lays, r = G.tune_multigraph(rp, col, od, voff, cache=cache, sweeps=4)
    assert r["from_cache"] and r["blocked"] and r["candidates"] == 1
    assert all(d["blocked"] and d["block_rows"] == 300 and d["tile_words"] == 1024
               for d in lays)
    with G.MultiGraph(rp, col, od, voff, layouts=lays) as mg:
        s, iters, _, _ = mg.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
        u, it_u, _, _ = mg.pagerank(tol=1e-6, max_iter=100, form=G.FORM_EXACT)
    assert np.all(np.abs(iters.astype(int) - it_u.astype(int)) <= 1)
    assert np.all(np.abs(s - u) <= 1e-6)
    with G.MultiGraph(rp, col, od, voff) as mg:  # no blocked layout: refused
        with pytest.raises(G.GprError):
            mg.pagerank(tol=1e-6, max_iter=100, form=G.FORM_BLOCKED)
