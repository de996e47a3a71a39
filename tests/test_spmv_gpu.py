"""CSR SpMV on the GPU through the C ABI, checked against the oracle.

Rows with at most 64 entries are summed with the reference's float
operations in the reference's order (src/spmv/omp_base.cc:18-28): the result
must be bit-identical.  Longer rows are summed as a tree: their error is
bounded by 1e-6 of the sum of |products|.  The 27-point stencil at full size
(128^3, 55.7M nonzeros) is checked bit-for-bit, which also meets the
reference verifier's maximum-relative-error criterion (<= 1e-6 here).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_stencil_small_bit_identical(G, O):
    Ap, Aj, Ax = O.stencil27(20)
    m = len(Ap) - 1
    x = O.uniform_f32(m, 5)
    for y0 in (np.zeros(m, np.float32), O.uniform_f32(m, 6)):
        y = y0.copy()
        G.SpmvSolver(m, len(Aj), Ap, Aj, Ax, x, y)
        assert np.array_equal(y, O.spmv_f32(Ap, Aj, Ax, x, y0))


def test_stencil_128_full_size(G, O):
    torch = pytest.importorskip("torch")
    A = G.gen_stencil27(128)
    assert A.m == 128 ** 3 and A.nnz == 382 ** 3
    x = torch.empty(A.m, dtype=torch.float32, device="cuda")
    G.gen_uniform(A.m, 11, x)
    y = torch.zeros(A.m, dtype=torch.float32, device="cuda")
    M = G.Matrix(A.rowptr, A.col, A.third, m=A.m, nnz=A.nnz)
    M.spmv(x, y)
    torch.cuda.synchronize()
    Ap, Aj, Ax = A.rowptr.to_numpy(), A.col.to_numpy(), A.third.to_numpy()
    xr = O.uniform_f32(A.m, 11)
    assert np.array_equal(x.cpu().numpy(), xr)
    yr = O.spmv_f32(Ap, Aj, Ax, xr, np.zeros(A.m, np.float32))
    yg = y.cpu().numpy()
    assert O.max_rel_err(yg, yr) <= 1e-6
    assert np.array_equal(yg, yr)
    M.close()
    A.close()


def test_long_and_ragged_rows(G, O):
    rng = np.random.default_rng(2)
    m = 3000
    lens = rng.integers(0, 20, m)
    lens[[0, 7, 100, 2999]] = [5000, 65, 64, 3000]
    lens[[1, 2]] = 0
    Ap = np.zeros(m + 1, np.int32)
    np.cumsum(lens, out=Ap[1:])
    Aj = np.concatenate([np.sort(rng.choice(m, size=l, replace=l > m)) for l in lens]).astype(np.int32)
    Ax = (1.0 - 2.0 * rng.random(len(Aj))).astype(np.float32)
    x = rng.random(m).astype(np.float32)
    y0 = rng.random(m).astype(np.float32)
    y = y0.copy()
    G.SpmvSolver(m, len(Aj), Ap, Aj, Ax, x, y)
    yr = O.spmv_f32(Ap, Aj, Ax, x, y0)
    short = lens <= 64
    assert np.array_equal(y[short], yr[short])
    absum = np.array([np.abs(x[Aj[Ap[i]:Ap[i + 1]]] * Ax[Ap[i]:Ap[i + 1]]).sum() + abs(y0[i])
                      for i in range(m)])
    assert np.all(np.abs(y - yr) <= 1e-6 * absum + 1e-30)


def test_empty_matrix(G):
    Ap = np.zeros(11, np.int32)
    y = np.arange(10, dtype=np.float32)
    G.SpmvSolver(10, 0, Ap, np.array([], np.int32), np.array([], np.float32),
                 np.ones(10, np.float32), y)
    assert np.array_equal(y, np.arange(10, dtype=np.float32))
