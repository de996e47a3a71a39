"""Multicolour symmetric Gauss-Seidel on the GPU, bit-identical to the
reference's SymGSSolver (fixtures made by the reference) and to the oracle's
restatement on larger stencils and several sweeps."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLD = os.path.join(ROOT, "tests", "golden")


def test_symgs_matches_reference_fixtures(G):
    gold = np.load(os.path.join(GOLD, "symgs.npz"))
    for g in sorted({k.split(":")[0] for k in gold.files}):
        a = {k: gold[f"{g}:{k}"] for k in ("Ap", "Aj", "Ax", "indices", "color_offsets", "x0",
                                           "b", "x")}
        x = a["x0"].copy()
        G.SymGSSolver(len(a["Ap"]) - 1, len(a["Aj"]), a["Ap"], a["Aj"], a["indices"], a["Ax"], x,
                      a["b"], a["color_offsets"])
        assert np.array_equal(x, a["x"]), g


@pytest.mark.parametrize("n", [2, 17, 40])
def test_symgs_stencil_several_sweeps(G, O, n):
    Ap, Aj, Ax = O.stencil27(n)
    m = len(Ap) - 1
    idx, co = O.greedy_coloring(Ap, Aj)
    x0, b = O.uniform_f32(m, 21), O.uniform_f32(m, 22)
    with G.SymGS(Ap, Aj, Ax, idx, co) as S:
        x = x0.copy()
        S.apply(x, b, sweeps=3)
    xr = x0
    for _ in range(3):
        xr = O.symgs_f32(Ap, Aj, Ax, idx, co, xr, b)
    assert np.array_equal(x, xr)


def test_symgs_rejects_invalid_colouring(G, O):
    Ap, Aj, Ax = O.stencil27(4)
    m = len(Ap) - 1
    idx = np.arange(m, dtype=np.int32)
    with pytest.raises(G.GprError) as e:
        G.SymGS(Ap, Aj, Ax, idx, np.array([0, m], np.int32))  # one colour for all
    assert e.value.status == G.GPR_EINVAL
    with pytest.raises(G.GprError) as e:
        bad = idx.copy()
        bad[1] = 0  # not a permutation
        G.SymGS(Ap, Aj, Ax, bad, np.array([0, m], np.int32))
    assert e.value.status == G.GPR_EINVAL


def test_symgs_zero_diagonal_rows_unchanged(G, O):
    # rows without a diagonal entry keep their x (src/symgs: diag != 0 test)
    Ap, Aj, Ax = O.stencil27(6)
    Ax = Ax.copy()
    Ax[Ax == 26.0] = 0.0
    Ax[: Ap[5]][Aj[: Ap[5]] == 0] = 0.0
    m = len(Ap) - 1
    idx, co = O.greedy_coloring(Ap, Aj)
    x0, b = O.uniform_f32(m, 1), O.uniform_f32(m, 2)
    x = x0.copy()
    G.SymGSSolver(m, len(Aj), Ap, Aj, idx, Ax, x, b, co)
    assert np.array_equal(x, x0)
