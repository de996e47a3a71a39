"""GPU input generators reproduce the oracle's generators bit-for-bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,ef,scramble", [(10, 16, True), (14, 8, False), (16, 16, True)])
def test_rmat_identical(G, O, scale, ef, scramble):
    g = G.gen_rmat(scale, ef, seed=1, scramble=scramble)
    rp, col, od = O.rmat_graph(scale, ef, seed=1, scramble=scramble)
    assert g.nnz == len(col)
    assert np.array_equal(g.rowptr.to_numpy(), rp)
    assert np.array_equal(g.col.to_numpy(), col)
    assert np.array_equal(g.third.to_numpy(), od)
    g.close()


@pytest.mark.parametrize("n", [1, 2, 9, 17])
def test_stencil_identical(G, O, n):
    A = G.gen_stencil27(n)
    Ap, Aj, Ax = O.stencil27(n)
    assert np.array_equal(A.rowptr.to_numpy(), Ap)
    assert np.array_equal(A.col.to_numpy(), Aj)
    assert np.array_equal(A.third.to_numpy(), Ax)
    A.close()
