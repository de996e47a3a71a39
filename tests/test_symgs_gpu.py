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


def test_symgs_stencil128_parity_colouring_full_size(G, O):
    """The benchmark's case: 27-point 128^3 stencil, 8-colour parity colouring,
    296 row domains synchronised only with their neighbours; two sweeps,
    bit-identical to the oracle's sequential colour order."""
    n = 128
    Ap, Aj, Ax = O.stencil27(n)
    m = len(Ap) - 1
    v = np.arange(m, dtype=np.int64)
    color = (v % n % 2) + 2 * ((v // n) % n % 2) + 4 * ((v // (n * n)) % 2)
    idx = np.argsort(color, kind="stable").astype(np.int32)
    co = np.zeros(9, dtype=np.int32)
    np.cumsum(np.bincount(color, minlength=8), out=co[1:])
    x0, b = O.uniform_f32(m, 31), O.uniform_f32(m, 32)
    with G.SymGS(Ap, Aj, Ax, idx, co) as S:
        x = x0.copy()
        S.apply(x, b, sweeps=2)
    xr = O.symgs_f32(Ap, Aj, Ax, idx, co, O.symgs_f32(Ap, Aj, Ax, idx, co, x0, b), b)
    assert np.array_equal(x, xr)


@pytest.mark.parametrize("seed", [1, 2])
def test_symgs_irregular_matrix(G, O, seed):
    """A random symmetric sparsity pattern with a few dense rows and a greedy
    colouring: domains of uneven row counts with many neighbours each."""
    rng = np.random.default_rng(seed)
    m = 60000
    src = rng.integers(0, m, 4 * m)
    dst = rng.integers(0, m, 4 * m)
    hubs = rng.integers(0, m, 20)
    src = np.concatenate([src, np.repeat(hubs, 3000), np.arange(m)])
    dst = np.concatenate([dst, rng.integers(0, m, 20 * 3000), np.arange(m)])
    a, c = np.concatenate([src, dst]), np.concatenate([dst, src])
    key = np.unique(a.astype(np.int64) * m + c)
    rows, cols = (key // m).astype(np.int32), (key % m).astype(np.int32)
    Ap = np.zeros(m + 1, dtype=np.int32)
    np.cumsum(np.bincount(rows, minlength=m), out=Ap[1:])
    Aj = cols
    Ax = np.where(rows == cols, np.float32(40.0),
                  rng.random(len(cols), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    idx, co = O.greedy_coloring(Ap, Aj)
    x0, b = O.uniform_f32(m, 5), O.uniform_f32(m, 6)
    with G.SymGS(Ap, Aj, Ax, idx, co) as S:
        x = x0.copy()
        S.apply(x, b, sweeps=2)
    xr = O.symgs_f32(Ap, Aj, Ax, idx, co, O.symgs_f32(Ap, Aj, Ax, idx, co, x0, b), b)
    assert np.array_equal(x, xr)
