"""ctypes bindings for the oracle (test infrastructure only).

It checks results; it is never the thing measured or shipped.  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import it; the product package ``gardenia_ocl_b200`` never does.

Two libraries are bound:

* ``liboracle.so`` -- the CPU restatement in ``oracle.c`` (plain FP32 PR
  after src/pr/omp_base.cc:9-49, FP64 fixed point, the push check of
  src/pr/verifier.cc:50-68, SpMV after src/spmv/omp_base.cc:8-32, the
  relative-error metric of src/spmv/verifier.cc:9-22, batched PPR, and the
  seeded generators).
* ``_ref/libgardenia_ref.so`` -- the reference's own OpenMP solvers,
  verifiers and ``read_graph`` compiled from the reference tree
  (``oracle/Makefile``).  Optional: absent on machines without the tree
  unless built beforehand.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

KDAMP = np.float32(0.85)  # include/common.h:18


def reference_root() -> str:
    """The reference tree the recipe in oracle/Makefile compiles from: its
    REF_ROOT (environment first, then the Makefile's default, the directory
    `reference` beside the repository's parent)."""
    env = os.environ.get("REF_ROOT")
    if env:
        return env
    return os.path.abspath(os.path.join(_HERE, "..", "..", "reference"))


def build() -> None:
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_pr_plain_f32.restype = C.c_int
        L.orc_pr_plain_f32.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f32p, C.c_float,
                                       C.c_double, C.c_int, C.c_void_p]
        L.orc_pr_f64.restype = C.c_int
        L.orc_pr_f64.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, C.c_float,
                                 C.c_double, C.c_int, C.POINTER(C.c_double)]
        L.orc_pr_residual_f64.restype = C.c_double
        L.orc_pr_residual_f64.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f32p, C.c_float]
        L.orc_err_vs_f64.restype = None
        L.orc_err_vs_f64.argtypes = [C.c_int, _f32p, _f64p, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]
        L.orc_pr_push_check.restype = C.c_double
        L.orc_pr_push_check.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f32p, C.c_float]
        L.orc_spmv_f32.restype = None
        L.orc_spmv_f32.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p]
        L.orc_max_rel_err_f32.restype = C.c_float
        L.orc_max_rel_err_f32.argtypes = [_f32p, _f32p, C.c_longlong]
        L.orc_ppr_f64.restype = None
        L.orc_ppr_f64.argtypes = [C.c_int, _i32p, _i32p, _i32p, C.c_int, _i32p, C.c_float,
                                  C.c_double, C.c_int, _f64p, _i32p]
        L.orc_rmat_edges.restype = None
        L.orc_rmat_edges.argtypes = [C.c_int, C.c_longlong, C.c_double, C.c_double,
                                     C.c_double, C.c_ulonglong, C.c_int, _i32p, _i32p]
        L.orc_build_in_csr.restype = C.c_longlong
        L.orc_build_in_csr.argtypes = [C.c_int, C.c_longlong, _i32p, _i32p, _i32p, _i32p, _i32p]
        L.orc_stencil27.restype = C.c_longlong
        L.orc_stencil27.argtypes = [C.c_int, _i32p, _i32p, _f32p]
        L.orc_uniform_f32.restype = None
        L.orc_uniform_f32.argtypes = [C.c_longlong, C.c_ulonglong, _f32p]
        L.orc_uniform_int.restype = None
        L.orc_uniform_int.argtypes = [C.c_longlong, C.c_ulonglong, C.c_int, _i32p]
        L.orc_num_threads.restype = C.c_int
        L.orc_symgs_f32.restype = None
        L.orc_symgs_f32.argtypes = [C.c_int, _i32p, _i32p, _f32p, _i32p, _i32p, C.c_int, _f32p,
                                    _f32p]
        L.orc_greedy_coloring.restype = C.c_int
        L.orc_greedy_coloring.argtypes = [C.c_int, _i32p, _i32p, _i32p]
        L.orc_multigraph_size.restype = C.c_int
        L.orc_multigraph_size.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong]
        L.orc_chung_lu_prefix.restype = None
        L.orc_chung_lu_prefix.argtypes = [C.c_int, C.c_double, _f64p]
        L.orc_multigraph_edges.restype = None
        L.orc_multigraph_edges.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, _f64p,
                                           _i32p, _i32p]
        _LIB = L
    return _LIB


def num_threads() -> int:
    return int(lib().orc_num_threads())


# --------------------------------------------------------------------------
# PageRank
# --------------------------------------------------------------------------
def pr_plain_f32(rowptr, col, outdeg, scores=None, tol=1e-3, max_iter=30,
                 damping=KDAMP):
    """Restated src/pr/omp_base.cc PRSolver.  Returns (scores, sweeps, err_hist)."""
    m = len(rowptr) - 1
    s = (np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
         if scores is None else np.ascontiguousarray(scores, dtype=np.float32).copy())
    hist = np.zeros(max(max_iter, 1), dtype=np.float64)
    n = lib().orc_pr_plain_f32(m, _c(rowptr), _c(col), _c(outdeg), s, float(damping),
                               float(tol), int(max_iter), hist.ctypes.data)
    return s, int(n), hist[:n].copy()


def pr_f64(rowptr, col, outdeg, tol=1e-14, max_iter=2000, damping=KDAMP, init=None):
    """FP64 fixed point of the plain recurrence.  Returns (scores_f64, sweeps, last_err)."""
    m = len(rowptr) - 1
    s = np.full(m, 1.0 / m, dtype=np.float64) if init is None else np.array(init, dtype=np.float64)
    err = C.c_double(0.0)
    n = lib().orc_pr_f64(m, _c(rowptr), _c(col), _c(outdeg), s, float(damping),
                         float(tol), int(max_iter), C.byref(err))
    return s, int(n), float(err.value)


def pr_residual_f64(rowptr, col, outdeg, scores, damping=KDAMP) -> float:
    m = len(rowptr) - 1
    return float(lib().orc_pr_residual_f64(m, _c(rowptr), _c(col), _c(outdeg),
                                           np.ascontiguousarray(scores, dtype=np.float32),
                                           float(damping)))


def err_vs_f64(a, ref):
    mx, l1 = C.c_double(), C.c_double()
    lib().orc_err_vs_f64(len(a), np.ascontiguousarray(a, dtype=np.float32),
                         np.ascontiguousarray(ref, dtype=np.float64), C.byref(mx), C.byref(l1))
    return float(mx.value), float(l1.value)


def push_check(out_rowptr, out_col, outdeg, scores, damping=KDAMP) -> float:
    """The L1 number PRVerifier compares against its target (verifier.cc:50-68)."""
    m = len(out_rowptr) - 1
    return float(lib().orc_pr_push_check(m, _c(out_rowptr), _c(out_col), _c(outdeg),
                                         np.ascontiguousarray(scores, dtype=np.float32),
                                         float(damping)))


def ppr_f64(rowptr, col, outdeg, seeds, tol=1e-6, max_iter=100, damping=KDAMP):
    m = len(rowptr) - 1
    k = len(seeds)
    x = np.zeros(m * k, dtype=np.float64)
    iters = np.zeros(k, dtype=np.int32)
    lib().orc_ppr_f64(m, _c(rowptr), _c(col), _c(outdeg), k, _c(seeds), float(damping),
                      float(tol), int(max_iter), x, iters)
    return x.reshape(m, k), iters


# --------------------------------------------------------------------------
# SpMV
# --------------------------------------------------------------------------
def spmv_f32(Ap, Aj, Ax, x, y):
    """Restated src/spmv/omp_base.cc SpmvSolver: returns y + A x (new array)."""
    out = np.ascontiguousarray(y, dtype=np.float32).copy()
    lib().orc_spmv_f32(len(Ap) - 1, _c(Ap), _c(Aj), _cf(Ax), _cf(x), out)
    return out


def max_rel_err(a, b) -> float:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return float(lib().orc_max_rel_err_f32(a, b, len(a)))


# --------------------------------------------------------------------------
# Generators
# --------------------------------------------------------------------------
RMAT_ABC = (0.57, 0.19, 0.19)


def rmat_edges(scale, edge_factor=16, seed=1, abc=RMAT_ABC, scramble=True):
    ne = (1 << scale) * edge_factor
    src = np.empty(ne, dtype=np.int32)
    dst = np.empty(ne, dtype=np.int32)
    lib().orc_rmat_edges(scale, ne, abc[0], abc[1], abc[2], seed, 1 if scramble else 0, src, dst)
    return src, dst


def in_csr_from_edges(m, src, dst):
    rowptr = np.empty(m + 1, dtype=np.int32)
    col = np.empty(len(src), dtype=np.int32)
    outdeg = np.empty(m, dtype=np.int32)
    nnz = lib().orc_build_in_csr(m, len(src), _c(src), _c(dst), rowptr, col, outdeg)
    return rowptr, col[:nnz].copy(), outdeg


def rmat_graph(scale, edge_factor=16, seed=1, abc=RMAT_ABC, scramble=True):
    """Seeded RMAT pull graph: (in_rowptr, in_col, outdeg), self-loops and
    duplicates removed, columns ascending within each row."""
    src, dst = rmat_edges(scale, edge_factor, seed, abc, scramble)
    return in_csr_from_edges(1 << scale, src, dst)


MULTI_ER_DEG, MULTI_CL_DEG, MULTI_GAMMA = 8, 16, 2.1


def multigraph(n_graphs, m_min=1000, m_max=500000, seed=1, er_deg=MULTI_ER_DEG,
               cl_deg=MULTI_CL_DEG, gamma=MULTI_GAMMA):
    """Seeded uneven batch of graphs as one block-diagonal pull graph
    (oracle.c orc_multigraph_*): graph g owns vertices [voff[g], voff[g+1]),
    odd g Chung-Lu power law (cl_deg draws per vertex, exponent gamma), even
    g Erdos-Renyi (er_deg draws per vertex).  Returns
    (in_rowptr, in_col, outdeg, voff) with global vertex ids."""
    L = lib()
    sizes = [int(L.orc_multigraph_size(g, m_min, m_max, seed)) for g in range(n_graphs)]
    voff = np.zeros(n_graphs + 1, dtype=np.int64)
    np.cumsum(sizes, out=voff[1:])
    P = np.empty(max(sizes) if sizes else 1, dtype=np.float64)
    L.orc_chung_lu_prefix(len(P), float(gamma), P)
    srcs, dsts = [], []
    for g, mg in enumerate(sizes):
        deg = cl_deg if g & 1 else er_deg
        s = np.empty(mg * deg, dtype=np.int32)
        d = np.empty(mg * deg, dtype=np.int32)
        L.orc_multigraph_edges(g, mg, deg, seed, P, s, d)
        srcs.append(s + np.int32(voff[g]))
        dsts.append(d + np.int32(voff[g]))
    M = int(voff[-1])
    src = np.concatenate(srcs) if srcs else np.zeros(0, np.int32)
    dst = np.concatenate(dsts) if dsts else np.zeros(0, np.int32)
    rp, col, od = in_csr_from_edges(M, src, dst)
    return rp, col, od, voff.astype(np.int32)


def stencil27(n):
    m = n ** 3
    cap = (3 * n - 2) ** 3
    Ap = np.empty(m + 1, dtype=np.int32)
    Aj = np.empty(cap, dtype=np.int32)
    Ax = np.empty(cap, dtype=np.float32)
    nnz = lib().orc_stencil27(n, Ap, Aj, Ax)
    assert nnz == cap
    return Ap, Aj, Ax


def uniform_f32(n, seed):
    out = np.empty(n, dtype=np.float32)
    lib().orc_uniform_f32(n, seed, out)
    return out


def uniform_int(n, seed, hi):
    out = np.empty(n, dtype=np.int32)
    lib().orc_uniform_int(n, seed, hi, out)
    return out


def csr_from_pushes(m, row, col, wt, sorted=True, remove_selfloops=True, remove_redundents=True):
    """fill_data of include/graph_io.h:21-130 over a push list (entry k
    appends (col[k], wt[k]) to the list of vertex row[k], in order): per-row
    lists in push order, optionally sorted by column (stable), self-loops
    dropped, then entries equal to the previous kept one dropped.  Returns
    (rowptr, col, wt)."""
    row = np.asarray(row, dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    wt = np.asarray(wt, dtype=np.float32)
    order = np.lexsort((col, row)) if sorted else np.argsort(row, kind="stable")
    r, c, w = row[order], col[order], wt[order]
    if remove_selfloops:
        keep = c != r
        r, c, w = r[keep], c[keep], w[keep]
    if remove_redundents and len(r):
        keep = np.ones(len(r), dtype=bool)
        keep[1:] = ~((r[1:] == r[:-1]) & (c[1:] == c[:-1]))
        r, c, w = r[keep], c[keep], w[keep]
    rowptr = np.zeros(m + 1, dtype=np.int32)
    np.cumsum(np.bincount(r, minlength=m), out=rowptr[1:])
    return rowptr, c.astype(np.int32), w


def greedy_coloring(rowptr, col):
    """First-fit colouring in vertex order; returns (indices, color_offsets):
    vertices sorted by colour (ties by id) and the colour boundaries, as the
    reference's SymGS driver builds them (src/symgs/main.cc:36-46)."""
    m = len(rowptr) - 1
    colors = np.empty(m, dtype=np.int32)
    nc = lib().orc_greedy_coloring(m, _c(rowptr), _c(col), colors)
    indices = np.argsort(colors, kind="stable").astype(np.int32)
    offsets = np.zeros(nc + 1, dtype=np.int32)
    np.cumsum(np.bincount(colors, minlength=nc), out=offsets[1:])
    return indices, offsets


def symgs_f32(rowptr, col, vals, indices, color_offsets, x, b):
    """One multicolour symmetric Gauss-Seidel sweep (src/symgs/verifier.cc
    gs_serial order); returns the new x."""
    m = len(rowptr) - 1
    xo = np.ascontiguousarray(x, dtype=np.float32).copy()
    lib().orc_symgs_f32(m, _c(rowptr), _c(col), _cf(vals), _c(indices), _c(color_offsets),
                        len(color_offsets) - 1, xo, _cf(b))
    return xo


def transpose_csr(m, rowptr, col):
    """Out-CSR of a pull (in-)CSR, columns ascending: used for the push check."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(rowptr))
    order = np.lexsort((rows, col))
    t_col = rows[order].astype(np.int32)
    cnt = np.bincount(col, minlength=m)
    t_ptr = np.zeros(m + 1, dtype=np.int32)
    np.cumsum(cnt, out=t_ptr[1:])
    return t_ptr, t_col


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref)
# --------------------------------------------------------------------------
def ref_path() -> str:
    return os.path.join(_HERE, "_ref", "libgardenia_ref.so")


def ref_available() -> bool:
    return os.path.exists(ref_path())


def ref():
    global _REF
    if _REF is None:
        R = C.CDLL(ref_path())
        R.ref_set_constants.argtypes = [C.c_double, C.c_int]
        R.ref_pr_solver.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _f32p]
        R.ref_pr_verifier.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _f32p, C.c_double]
        R.ref_spmv_solver.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p]
        R.ref_spmv_verifier.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p]
        R.ref_read_graph.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int)),
                                     C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_float))]
        R.ref_free.argtypes = [C.c_void_p]
        R.ref_symgs_solver.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _i32p, _f32p, _f32p, _f32p,
                                       _i32p, C.c_int]
        _REF = R
    return _REF


class _CaptureStdout:
    """Redirect the process's fd 1 (C stdio) into a temp file."""

    def __enter__(self):
        self._tmp = tempfile.TemporaryFile(mode="w+b")
        self._saved = os.dup(1)
        os.dup2(self._tmp.fileno(), 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self._saved, 1)
        os.close(self._saved)
        self._tmp.seek(0)
        self.text = self._tmp.read().decode(errors="replace")
        self._tmp.close()
        return False


def ref_pr_solver(in_rowptr, in_col, outdeg, scores=None, tol=1e-3, max_iter=30,
                  out_rowptr=None, out_col=None):
    """Run the reference PRSolver.  Returns (scores, printed_iterations, stdout).

    The printed iteration count is ``iter+1`` (src/pr/omp_base.cc:46): the
    number of sweeps when it converged, max_iter+1 when it did not."""
    m = len(in_rowptr) - 1
    nnz = len(in_col)
    s = (np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
         if scores is None else np.ascontiguousarray(scores, dtype=np.float32).copy())
    orp = _c(out_rowptr) if out_rowptr is not None else _c(in_rowptr)
    oc = _c(out_col) if out_col is not None else _c(in_col)
    R = ref()
    R.ref_set_constants(float(tol), int(max_iter))
    with _CaptureStdout() as cap:
        R.ref_pr_solver(m, nnz, _c(in_rowptr), _c(in_col), orp, oc, _c(outdeg), s)
    it = re.search(r"iterations = (\d+)", cap.text)
    return s, (int(it.group(1)) if it else -1), cap.text


def ref_pr_verifier(in_rowptr, in_col, out_rowptr, out_col, outdeg, scores,
                    target=1e-3, max_iter=30):
    m = len(in_rowptr) - 1
    R = ref()
    R.ref_set_constants(float(target), int(max_iter))
    with _CaptureStdout() as cap:
        R.ref_pr_verifier(m, _c(in_rowptr), _c(in_col), _c(out_rowptr), _c(out_col),
                          _c(outdeg), np.ascontiguousarray(scores, dtype=np.float32), float(target))
    return cap.text


def ref_spmv_solver(Ap, Aj, Ax, x, y):
    out = np.ascontiguousarray(y, dtype=np.float32).copy()
    with _CaptureStdout() as cap:
        ref().ref_spmv_solver(len(Ap) - 1, len(Aj), _c(Ap), _c(Aj), _cf(Ax), _cf(x), out)
    return out, cap.text


def ref_symgs_solver(rowptr, col, vals, indices, color_offsets, x, b):
    """The reference's OpenMP SymGSSolver (src/symgs/omp_base.cc); returns
    (x, stdout)."""
    R = ref()
    xo = np.ascontiguousarray(x, dtype=np.float32).copy()
    co = _c(color_offsets)
    with _CaptureStdout() as cap:
        R.ref_symgs_solver(len(rowptr) - 1, len(col), _c(rowptr), _c(col), _c(indices),
                           _cf(vals), xo, _cf(b), co, len(co))
    return xo, cap.text


_REF_GPU = {}


def ref_gpu_available(name="gather") -> bool:
    """The reference's own CUDA solver `name` (gather, gather_warp, spmv_base),
    recompiled for sm_100a into oracle/_ref."""
    return os.path.exists(os.path.join(_HERE, "_ref", f"libgardenia_ref_{name}.so"))


def _ref_gpu(name):
    if name not in _REF_GPU:
        R = C.CDLL(os.path.join(_HERE, "_ref", f"libgardenia_ref_{name}.so"))
        R.ref_set_constants.argtypes = [C.c_double, C.c_int]
        if name.startswith("gather"):
            R.ref_gpu_pr_solver.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _i32p, _f32p]
        else:
            R.ref_gpu_spmv_solver.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p]
        _REF_GPU[name] = R
    return _REF_GPU[name]


def _runtime_ms(text):
    import re
    mt = re.search(r"runtime \[[^\]]*\] = ([0-9.]+) ms", text)
    return float(mt.group(1)) if mt else float("nan")


def ref_gpu_pr_solver(name, rowptr, col, outdeg, scores=None, tol=1e-3, max_iter=30):
    """The reference's CUDA PRSolver (src/pr/gather.cu or gather_warp.cu) on the
    GPU: returns (scores, sweeps, runtime_ms of its own Timer, stdout)."""
    import re
    R = _ref_gpu(name)
    m = len(rowptr) - 1
    s = (np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32) if scores is None
         else np.ascontiguousarray(scores, dtype=np.float32).copy())
    R.ref_set_constants(float(tol), int(max_iter))
    with _CaptureStdout() as cap:
        R.ref_gpu_pr_solver(m, len(col), _c(rowptr), _c(col), _c(outdeg), s)
    it = re.search(r"iterations = (\d+)\.", cap.text)
    return s, int(it.group(1)) if it else -1, _runtime_ms(cap.text), cap.text


def ref_gpu_spmv_solver(Ap, Aj, Ax, x, y):
    """The reference's CUDA SpmvSolver (src/spmv/base.cu): returns (y, runtime_ms)."""
    R = _ref_gpu("spmv_base")
    yo = np.ascontiguousarray(y, dtype=np.float32).copy()
    with _CaptureStdout() as cap:
        R.ref_gpu_spmv_solver(len(Ap) - 1, len(Aj), _c(Ap), _c(Aj), _cf(Ax), _cf(x), yo)
    return yo, _runtime_ms(cap.text)


def ref_read_graph(path, symmetrize=False, transpose=False, sorted=True,
                   remove_selfloops=True, remove_redundents=True):
    """The reference loader (include/graph_io.h:280).  Returns
    (rowptr, col, degree, weight, stdout)."""
    R = ref()
    m, nnz = C.c_int(), C.c_int()
    rp, cp, dp = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    wp = C.POINTER(C.c_float)()
    with _CaptureStdout() as cap:
        R.ref_read_graph(path.encode(), int(symmetrize), int(transpose), int(sorted),
                         int(remove_selfloops), int(remove_redundents), C.byref(m), C.byref(nnz),
                         C.byref(rp), C.byref(cp), C.byref(dp), C.byref(wp))
    mm, nz = m.value, nnz.value
    rowptr = np.ctypeslib.as_array(rp, shape=(mm + 1,)).copy()
    col = np.ctypeslib.as_array(cp, shape=(max(nz, 1),))[:nz].copy()
    deg = np.ctypeslib.as_array(dp, shape=(max(mm, 1),))[:mm].copy()
    wt = np.ctypeslib.as_array(wp, shape=(max(nz, 1),))[:nz].copy()
    for p in (rp, cp, dp, wp):
        R.ref_free(C.cast(p, C.c_void_p))
    return rowptr, col, deg, wt, cap.text


def _c(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _cf(a):
    return np.ascontiguousarray(a, dtype=np.float32)
