"""The reference's own PR driver (src/pr/main.cc, unmodified) linked against
libgpr.so instead of a reference solver object: the link-time drop-in.

oracle/Makefile builds oracle/_ref/pr_gpr_dropin from the reference tree; the
driver reads the graph with the reference's own graph_io.h, calls libgpr's
PRSolver and PRVerifier, and must print the reference's lines: the same
sweep count as the reference's OpenMP solver on that file (golden fixture)
and the verifier verdict the reference's own scores get.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "pr_gpr_dropin")
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.mark.skipif(not os.path.exists(BIN), reason="drop-in driver not built (needs the reference tree at build time)")
@pytest.mark.parametrize("name", ["graph_small.mtx", "graph_dups.mtx", "graph_simple.mtx"])
@pytest.mark.parametrize("tol,max_iter", [(1e-3, 30), (1e-4, 100)])
def test_reference_driver_runs_on_libgpr(O, name, tol, max_iter):
    pr = np.load(os.path.join(GOLD, "pr.npz"))
    ld = np.load(os.path.join(GOLD, "loader.npz"))
    env = dict(os.environ, GPR_TOL=str(tol), GPR_MAX_ITER=str(max_iter))
    out = subprocess.run([BIN, os.path.join(GOLD, name)], capture_output=True, text=True,
                         timeout=300, env=env)
    assert out.returncode == 0, out.stderr
    assert "Launching B200 PR solver" in out.stdout
    sweeps = int(re.search(r"iterations = (\d+)\.", out.stdout).group(1))
    printed = int(pr[f"{name}:{tol:g}:{max_iter}:printed_iterations"][0])
    # the reference prints iter+1, which equals the sweeps when it converged
    assert sweeps in (printed, printed - 1)
    # PR driver flags: unsorted, self-loops and adjacent duplicates removed
    key = f"{name}:00011"
    ok = O.push_check(ld[key + ":rowptr"], ld[key + ":col"], pr[f"{name}:outdeg"],
                      pr[f"{name}:{tol:g}:{max_iter}:scores"]) < 1e-3
    assert ("Correct" in out.stdout) == ok


@pytest.mark.parametrize("name", ["test_pr.mtx", "chesapeake.mtx", "graph_small.mtx",
                                  "graph_dups.mtx", "graph_simple.mtx"])
@pytest.mark.parametrize("tol,max_iter", [(1e-3, 30), (1e-4, 100)])
def test_prsolver_scores_match_reference(G, O, capfd, monkeypatch, name, tol, max_iter):
    """libgpr's PRSolver symbol (src/pr/pr.h:23) called directly on the graphs
    the reference solved: its scores equal the reference's scores (golden
    fixture) within 1e-6, and bit for bit the oracle's at the same sweep
    count (every row of these graphs has at most 64 in-edges)."""
    import ctypes as C
    pr = np.load(os.path.join(GOLD, "pr.npz"))
    rp, col, od = (np.ascontiguousarray(pr[f"{name}:{k}"], dtype=np.int32)
                   for k in ("in_rowptr", "in_col", "outdeg"))
    m, nnz = len(rp) - 1, len(col)
    orp, ocol = (np.ascontiguousarray(a, dtype=np.int32) for a in O.transpose_csr(m, rp, col))
    s = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
    monkeypatch.setenv("GPR_TOL", str(tol))
    monkeypatch.setenv("GPR_MAX_ITER", str(max_iter))
    lib = C.CDLL(G.LIB_PATH)
    fn = getattr(lib, "_Z8PRSolveriiPiS_S_S_S_Pf")
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    fn(C.c_int(m), C.c_int(nnz), P(rp), P(col), P(orp), P(ocol), P(od), P(s))
    C.CDLL(None).fflush(None)
    out = capfd.readouterr().out
    sweeps = int(re.search(r"iterations = (\d+)\.", out).group(1))
    ref = pr[f"{name}:{tol:g}:{max_iter}:scores"]
    assert np.abs(s - ref).max() <= 1e-6
    exact, _, _ = O.pr_plain_f32(rp, col, od, tol=0.0, max_iter=sweeps)
    assert np.array_equal(s, exact)
