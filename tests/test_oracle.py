"""CPU: the oracle and the host-side loader, pinned to the reference itself.

The fixtures under tests/golden/ were produced by the reference's own code
(tests/golden/make_golden.py runs oracle/_ref, compiled from the reference
tree).  These tests hold everything a GPU result is compared against to
those fixtures bit for bit, and, where the reference tree is present, also
to the live reference on fresh seeded inputs.
"""
import itertools
import os

import numpy as np
import pytest

from conftest import ROOT

import oracle  # noqa: E402  (on sys.path through conftest)

GOLD = os.path.join(ROOT, "tests", "golden")
REF_DATA = os.path.join(oracle.reference_root(), "datasets")


@pytest.fixture(scope="module")
def pr_gold():
    return np.load(os.path.join(GOLD, "pr.npz"))


@pytest.fixture(scope="module")
def spmv_gold():
    return np.load(os.path.join(GOLD, "spmv.npz"))


@pytest.fixture(scope="module")
def loader_gold():
    return np.load(os.path.join(GOLD, "loader.npz"))


def graphs(d):
    return sorted({k.split(":")[0] for k in d.files})


def test_pr_restatement_bit_identical_to_reference(O, pr_gold):
    names = graphs(pr_gold)
    assert {"test_pr.mtx", "chesapeake.mtx", "4.mtx", "4.graph", "rmat10"} <= set(names)
    for g in names:
        rp, col, od = (pr_gold[f"{g}:{k}"] for k in ("in_rowptr", "in_col", "outdeg"))
        for tol, mi in ((1e-3, 30), (1e-4, 100)):
            s, sweeps, hist = O.pr_plain_f32(rp, col, od, tol=tol, max_iter=mi)
            gold = pr_gold[f"{g}:{tol:g}:{mi}:scores"]
            printed = int(pr_gold[f"{g}:{tol:g}:{mi}:printed_iterations"][0])
            assert np.array_equal(s, gold), g
            # omp_base.cc:46 prints iter+1: the sweep count when it converged,
            # max_iter+1 when it ran out of sweeps.
            converged = hist[-1] < tol
            assert printed == (sweeps if converged else sweeps + 1), g


def test_spmv_restatement_bit_identical_to_reference(O, spmv_gold):
    for g in graphs(spmv_gold):
        a = {k: spmv_gold[f"{g}:{k}"] for k in ("Ap", "Aj", "Ax", "x", "y0", "y")}
        y = O.spmv_f32(a["Ap"], a["Aj"], a["Ax"], a["x"], a["y0"])
        assert np.array_equal(y, a["y"]), g
        assert O.max_rel_err(y, a["y"]) == 0.0


def test_rmat_generator_is_pinned(O, pr_gold):
    rp, col, od = O.rmat_graph(10, 16, seed=1)
    assert np.array_equal(rp, pr_gold["rmat10:in_rowptr"])
    assert np.array_equal(col, pr_gold["rmat10:in_col"])
    assert np.array_equal(od, pr_gold["rmat10:outdeg"])


def test_reference_verifier_on_reference_scores(O, pr_gold, loader_gold):
    # PRVerifier's push check (src/pr/verifier.cc:50-68) on the reference's
    # own results for its datasets: the number it compares with EPSILON.
    # 4.mtx holds non-adjacent duplicate edges; the PR driver reads it
    # unsorted (src/pr/main.cc:23-24), so the out-CSR and the in-CSR keep
    # different duplicates and the reference fails its own check there.
    for ds, ok in (("test_pr.mtx", True), ("chesapeake.mtx", True), ("4.mtx", False),
                   ("4.graph", True)):
        orp, ocol = loader_gold[f"ref:{ds}:out_rowptr"], loader_gold[f"ref:{ds}:out_col"]
        od = pr_gold[f"{ds}:outdeg"]
        s = pr_gold[f"{ds}:0.001:30:scores"]
        assert (O.push_check(orp, ocol, od, s) < 1e-3) == ok, ds


def test_fp64_oracle_is_a_fixed_point(O, pr_gold):
    rp, col, od = (pr_gold[f"rmat10:{k}"] for k in ("in_rowptr", "in_col", "outdeg"))
    s64, n, err = O.pr_f64(rp, col, od)
    assert err < 1e-14
    # the FP32 result at tol 1e-4 lies within the a-posteriori bound of the fixed point
    s32 = pr_gold["rmat10:0.0001:100:scores"]
    r = O.pr_residual_f64(rp, col, od, s32)
    mx, l1 = O.err_vs_f64(s32, s64)
    assert l1 <= r / (1 - 0.85) * 1.0001 + 1e-12


@pytest.mark.parametrize("name", ["graph_small", "graph_dups", "graph_simple"])
@pytest.mark.parametrize("ext", [".mtx", ".gr", ".graph"])
def test_read_graph_matches_reference_loader(G, loader_gold, name, ext):
    path = os.path.join(GOLD, name + ext)
    for fl in itertools.product([False, True], repeat=5):
        key = name + ext + ":" + "".join(str(int(x)) for x in fl)
        m, nnz, rp, col, deg, wt = G.read_graph(path, *fl)
        assert np.array_equal(rp, loader_gold[key + ":rowptr"]), key
        assert np.array_equal(col, loader_gold[key + ":col"]), key
        assert np.array_equal(wt, loader_gold[key + ":weight"]), key
        assert np.array_equal(deg, np.diff(rp)), key


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference datasets not present")
@pytest.mark.parametrize("ds", ["test_pr.mtx", "chesapeake.mtx", "4.mtx", "4.graph"])
def test_read_graph_on_reference_datasets(G, loader_gold, ds):
    path = os.path.join(REF_DATA, ds)
    _, _, orp, ocol, _, _ = G.read_graph(path, False, False, False)
    _, _, irp, icol, _, _ = G.read_graph(path, False, True, False)
    assert np.array_equal(orp, loader_gold[f"ref:{ds}:out_rowptr"])
    assert np.array_equal(ocol, loader_gold[f"ref:{ds}:out_col"])
    assert np.array_equal(irp, loader_gold[f"ref:{ds}:in_rowptr"])
    assert np.array_equal(icol, loader_gold[f"ref:{ds}:in_col"])


def test_live_reference_on_fresh_graphs(O):
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    from graphs import erdos_renyi
    for seed in range(3):
        rp, col, od = erdos_renyi(3000, 7, seed=seed)
        a, na, _ = O.pr_plain_f32(rp, col, od, tol=1e-5, max_iter=60)
        b, nb, _ = O.ref_pr_solver(rp, col, od, tol=1e-5, max_iter=60)
        assert np.array_equal(a, b) and (nb == na or nb == na + 1)
        x = O.uniform_f32(3000, seed + 10)
        vals = O.uniform_f32(len(col), seed + 20)
        y0 = np.zeros(3000, np.float32)
        assert np.array_equal(O.spmv_f32(rp, col, vals, x, y0),
                              O.ref_spmv_solver(rp, col, vals, x, y0)[0])


def test_multigraph_generator_properties(O):
    rp, col, od, voff = O.multigraph(16, 1000, 50000, seed=1)
    sizes = np.diff(voff)
    assert sizes.min() >= 1000 and sizes.max() <= 50000
    m = len(rp) - 1
    assert voff[-1] == m and np.array_equal(od, np.bincount(col, minlength=m))
    for g in range(16):
        a, b = voff[g], voff[g + 1]
        c = col[rp[a]:rp[b]]
        assert c.min() >= a and c.max() < b  # block-diagonal
        deg = np.diff(rp[a:b + 1])
        avg = (rp[b] - rp[a]) / (b - a)
        if g % 2 == 0:  # Erdos-Renyi, 8 draws per vertex, few collisions
            assert 7.5 < avg <= 8.0 and deg.max() < 40
        else:           # Chung-Lu power law, 16 draws per vertex
            assert avg < 16.0 and deg.max() > 30 * avg
    for g in range(m and 16):
        r = rp[voff[g]:voff[g + 1] + 1]
        for v in range(0, len(r) - 1, 97):  # columns ascending, no self-loops
            cc = col[r[v]:r[v + 1]]
            assert np.all(np.diff(cc) > 0) and not np.any(cc == voff[g] + v)


def test_multigraph_sizes_log_uniform(O):
    L = O.lib()
    sizes = np.array([L.orc_multigraph_size(g, 1000, 500000, 7) for g in range(4000)])
    assert sizes.min() >= 1000 and sizes.max() <= 500000
    frac = np.mean(np.log(sizes) < 0.5 * (np.log(1000) + np.log(500000)))
    assert abs(frac - 0.5) < 0.03


def same_weights_per_entry(rp, c, w, w_ref):
    """Equal (row, column, weight) multisets: the weights of equal columns in
    a row may come in another order."""
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    a = np.lexsort((w, c, rows))
    b = np.lexsort((w_ref, c, rows))
    return np.array_equal(w[a], w_ref[b])


@pytest.mark.parametrize("name", ["graph_small", "graph_dups", "graph_simple"])
@pytest.mark.parametrize("ext", [".mtx", ".gr", ".graph"])
@pytest.mark.parametrize("threads", [1, 3, 8])
def test_parallel_parse_reproduces_reference_lists(G, O, loader_gold, name, ext, threads):
    # Pushes from the multithreaded parser, formed into lists by fill_data's
    # rules, give the reference loader's CSR under every flag combination.
    # With `sorted` the reference orders equal columns of a row by std::sort,
    # whose order among equal keys the C++ standard leaves unspecified; a
    # stable sort gives the same rows and columns, and the same weights except
    # that duplicate columns may carry them in another order (and duplicate
    # removal may then keep another duplicate's weight).
    path = os.path.join(GOLD, name + ext)
    for sym, trans in itertools.product([False, True], repeat=2):
        m, _, row, col, wt = G.parse_edges(path, sym, trans, threads=threads)
        for srt, sl, rd in itertools.product([False, True], repeat=3):
            key = name + ext + ":" + "".join(str(int(x)) for x in (sym, trans, srt, sl, rd))
            rp, c, w = O.csr_from_pushes(m, row, col, wt, srt, sl, rd)
            assert np.array_equal(rp, loader_gold[key + ":rowptr"]), key
            assert np.array_equal(c, loader_gold[key + ":col"]), key
            if not srt:
                assert np.array_equal(w, loader_gold[key + ":weight"]), key
            elif not rd:
                assert same_weights_per_entry(rp, c, w, loader_gold[key + ":weight"]), key


def test_symgs_restatement_bit_identical_to_reference(O):
    # src/symgs/omp_base.cc SymGSSolver, one sweep, fixtures made by the reference
    gold = np.load(os.path.join(GOLD, "symgs.npz"))
    for g in graphs(gold):
        a = {k: gold[f"{g}:{k}"] for k in ("Ap", "Aj", "Ax", "indices", "color_offsets", "x0",
                                           "b", "x")}
        idx, co = O.greedy_coloring(a["Ap"], a["Aj"])
        assert np.array_equal(idx, a["indices"]) and np.array_equal(co, a["color_offsets"]), g
        x = O.symgs_f32(a["Ap"], a["Aj"], a["Ax"], a["indices"], a["color_offsets"], a["x0"], a["b"])
        assert np.array_equal(x, a["x"]), g


@pytest.mark.parametrize("ext", [".mtx", ".gr"])
def test_parse_falls_back_on_irregular_lines(G, O, tmp_path, ext):
    # An entry line with missing numbers makes the reference reuse the values
    # left by the previous line -- already decremented in place, so they are
    # decremented once more (graph_io.h:155-158, :238-245).  The parallel
    # parser hands such files to the sequential reader, which reproduces it.
    p = tmp_path / ("irregular" + ext)
    if ext == ".mtx":
        p.write_text("%%MatrixMarket matrix coordinate real general\n5 5 6\n1 2 0.5\n3 4\n"
                     "\n4 5 -2\n5 1 1.5\n3 3 1\n")
    else:
        p.write_text("p sp 5 6\na 1 2 1\na 3 4 1\na\na 4 5 1\na 5 1 1\na 3 3 1\n")
    m, nnz, row, col, wt = G.parse_edges(str(p), threads=4)
    assert (m, nnz) == (5, 6) and len(row) == 6
    # the line without numbers repeats the previous edge decremented again
    assert list(zip(row, col)) == [(0, 1), (2, 3), (1, 2), (3, 4), (4, 0), (2, 2)]
    if ext == ".mtx":
        assert list(wt) == [0.5, 1.0, 1.0, 2.0, 1.5, 1.0]
    for fl in itertools.product([False, True], repeat=3):
        mm, nz, rp_ref, col_ref, deg, w_ref = G.read_graph(str(p), False, False, *fl)
        rp, c, w = O.csr_from_pushes(m, row, col, wt, *fl)
        assert np.array_equal(rp, rp_ref) and np.array_equal(c, col_ref)
        if O.ref_available():  # the reference's own loader on the same file
            rr, cr, _, wr, _ = O.ref_read_graph(str(p), False, False, *fl)
            assert np.array_equal(rp, rr) and np.array_equal(c, cr)
