"""The reference's own CUDA solvers (src/pr/gather.cu, gather_warp.cu,
src/spmv/base.cu), recompiled for sm_100a into oracle/_ref, beside this
library on the same B200: the results agree, and the timings of both are
printed (run with -s to see them).  The reference's solvers time their sweep
loop with their own Timer, which includes a device-to-host copy of the
residual after every sweep, as the reference's PR driver measures it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["gather", "gather_warp"])
def test_reference_cuda_pagerank_beside_ours(G, O, variant):
    if not O.ref_gpu_available(variant):
        pytest.skip("oracle/_ref CUDA solvers not built (needs the reference tree)")
    rp, col, od = O.rmat_graph(20, 16, seed=1)
    sweeps = 20
    ref, it, ref_ms, _ = O.ref_gpu_pr_solver(variant, rp, col, od, tol=0.0, max_iter=sweeps)
    assert it == sweeps
    with G.Graph(rp, col, od) as g:
        g.pagerank(tol=0.0, max_iter=sweeps)  # warm
        s, st = g.pagerank(tol=0.0, max_iter=sweeps)
    assert st.iterations == sweeps
    # the reference's kernel contracts base + kDamp*sum into one FMA; both
    # stay within 1e-6 of each other plus the float error of long rows
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=sweeps)
    assert np.all(np.abs(s - ref) <= 1e-6 + np.abs(ref - s64) + np.abs(s - s64))
    gteps_ref = len(col) * sweeps / (ref_ms / 1e3) / 1e9
    gteps = len(col) * sweeps / (st.solve_ms / 1e3) / 1e9
    print(f"\nRMAT s20, {sweeps} sweeps: reference {variant} {ref_ms:.2f} ms "
          f"({gteps_ref:.1f} GTEPS); gpr {st.solve_ms:.2f} ms ({gteps:.1f} GTEPS), "
          f"{gteps / gteps_ref:.1f}x")
    assert gteps > gteps_ref


def test_reference_cuda_spmv_beside_ours(G, O):
    if not O.ref_gpu_available("spmv_base"):
        pytest.skip("oracle/_ref CUDA solvers not built (needs the reference tree)")
    Ap, Aj, Ax = O.stencil27(96)
    m = len(Ap) - 1
    x, y0 = O.uniform_f32(m, 5), np.zeros(m, np.float32)
    yr, ref_ms = O.ref_gpu_spmv_solver(Ap, Aj, Ax, x, y0)
    y = y0.copy()
    G.SpmvSolver(m, len(Aj), Ap, Aj, Ax, x, y)
    # The reference's kernel contracts each row's multiply-adds into FMAs;
    # the stencil's rows cancel (26 x_i minus the neighbours), so compare
    # against the size of the terms: 1e-6 of each row's sum of |products|.
    rows = np.repeat(np.arange(m), np.diff(Ap))
    absum = np.bincount(rows, weights=np.abs(Ax * x[Aj]), minlength=m)
    assert np.all(np.abs(y - yr) <= 1e-6 * absum)
    # kernel time beside the reference's Timer (one launch + synchronize)
    import time
    A = G.Matrix(Ap, Aj, Ax)
    dx = G.DeviceArray(0, 0, np.float32)
    p = G.C.c_void_p()
    G.lib().gpr_malloc(G.C.byref(p), 8 * m)
    xd, yd = p.value, p.value + 4 * m
    G.lib().gpr_memcpy(G.C.c_void_p(xd), G.C.c_void_p(x.ctypes.data), 4 * m)
    G.lib().gpr_memcpy(G.C.c_void_p(yd), G.C.c_void_p(y0.ctypes.data), 4 * m)
    xa, ya = G.DeviceArray(xd, m, np.float32), G.DeviceArray(yd, m, np.float32)
    A.spmv(xa, ya)
    G.synchronize()
    t0 = time.perf_counter()
    for _ in range(20):
        A.spmv(xa, ya)
    G.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / 20
    xa.ptr = ya.ptr = 0  # one allocation, released below
    G.lib().gpr_free(G.C.c_void_p(xd))
    A.close()
    del dx
    print(f"\n27-point 96^3 SpMV: reference base {ref_ms:.3f} ms (its Timer, one launch); "
          f"gpr {ms:.3f} ms per launch, {ref_ms / ms:.1f}x")
    assert ms < ref_ms
