"""The verifiers libgpr exports under the reference's names give the
reference's verdicts: "Correct" on a result the oracle computed, a failure
line on a perturbed one.  They run on the host, so this is a CPU test: a
small C++ driver (tests/verifier_driver.cc) linked against libgpr calls them.

  PRVerifier    src/pr/verifier.cc:50-68   "Correct" / "Total Error: ..."
  SpmvVerifier  src/spmv/verifier.cc:55-61 "Correct" / "POSSIBLE FAILURE"
                (max relative error <= 5*sqrt(FLT_EPSILON))
  SymGSVerifier src/symgs/verifier.cc:82-90 "Correct" / "POSSIBLE FAILURE"
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def driver(G, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("drv") / "verifier_driver")
    libdir = os.path.dirname(G.LIB_PATH)
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-o", out,
                    os.path.join(ROOT, "tests", "verifier_driver.cc"),
                    "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lgpr",
                    "-Wl,-rpath," + libdir], check=True)
    return out


def run(driver, kind, d, arrays):
    for name, a in arrays.items():
        np.ascontiguousarray(a).tofile(os.path.join(d, name + ".bin"))
    p = subprocess.run([driver, kind, str(d)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    return p.stdout


def verdict(out):
    last = [l for l in out.splitlines() if l.strip()][-1]
    return last


def test_spmv_verifier_verdicts(driver, O, tmp_path):
    Ap, Aj, Ax = O.stencil27(12)
    m = len(Ap) - 1
    x = O.uniform_f32(m, 3)
    y = O.uniform_f32(m, 4)
    ty = O.spmv_f32(Ap, Aj, Ax, x, y.copy())
    base = dict(Ap=Ap, Aj=Aj, Ax=Ax, x=x, y=y)
    assert verdict(run(driver, "spmv", tmp_path, dict(base, test_y=ty))) == "Correct"
    # within the reference's bound (1e-4 relative < 5*sqrt(FLT_EPSILON)): still correct
    small = ty.copy()
    small[7] *= np.float32(1 + 1e-4)
    assert verdict(run(driver, "spmv", tmp_path, dict(base, test_y=small))) == "Correct"
    bad = ty.copy()
    bad[m // 2] *= np.float32(1.01)
    out = run(driver, "spmv", tmp_path, dict(base, test_y=bad))
    assert verdict(out) == "POSSIBLE FAILURE"
    assert "[max error" in out


def test_symgs_verifier_verdicts(driver, O, tmp_path):
    Ap, Aj, Ax = O.stencil27(10)
    m = len(Ap) - 1
    idx, co = O.greedy_coloring(Ap, Aj)
    b = O.uniform_f32(m, 4)
    x0 = O.uniform_f32(m, 5)
    tx = O.symgs_f32(Ap, Aj, Ax, idx, co, x0, b)
    base = dict(Ap=Ap, Aj=Aj, Ax=Ax, indices=idx, color_offsets=np.asarray(co, np.int32), x=x0, b=b)
    assert verdict(run(driver, "symgs", tmp_path, dict(base, test_x=tx))) == "Correct"
    bad = tx.copy()
    bad[m // 3] += np.float32(0.5)
    out = run(driver, "symgs", tmp_path, dict(base, test_x=bad))
    assert verdict(out) == "POSSIBLE FAILURE"
    assert f"x_test[{m // 3}]" in out


def test_pr_verifier_verdicts(driver, O, tmp_path):
    rp, col, od = O.rmat_graph(10, 8, seed=3)
    m = len(rp) - 1
    orp, ocol = O.transpose_csr(m, rp, col)
    s, n, _ = O.pr_plain_f32(rp, col, od, tol=1e-6, max_iter=200)
    base = dict(in_rowptr=rp, in_col=col, out_rowptr=orp, out_col=ocol, outdeg=od,
                target=np.array([1e-4]))
    assert verdict(run(driver, "pr", tmp_path, dict(base, scores=s))) == "Correct"
    bad = s.copy()
    bad[:m // 2] *= np.float32(1.5)
    assert verdict(run(driver, "pr", tmp_path, dict(base, scores=bad))).startswith("Total Error:")
