"""gardenia_ocl_b200 -- B200-native pull PageRank and CSR SpMV.

Python mirror of the reference's driver surface (Gardenia ``src/pr``,
``src/spmv``): ``PRSolver``, ``PageRank``, ``SpmvSolver``, ``read_graph``, plus
handle-based access (``Graph``, ``Matrix``) for device-resident, repeated
solves.  Every call goes through the C ABI of ``libgpr.so`` (include/gpr.h),
whose kernels are compiled for sm_100a; there is no CPU implementation of the
solvers in this package, and importing it on a machine without the built
library raises.

Arrays may be numpy arrays (host) or objects exposing ``data_ptr()`` (e.g.
torch CUDA tensors, device memory): the library copies host inputs itself.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgpr.so")

GPR_OK, GPR_EINVAL, GPR_ENOMEM, GPR_ECUDA, GPR_ETIMEOUT, GPR_ENODEV, GPR_EUNSUPPORTED = range(7)
PREC_FP32, PREC_BF16, PREC_FP16 = 0, 1, 2
LOOP_AUTO, LOOP_PERSISTENT, LOOP_GRAPH = 0, 1, 2
FORM_AUTO, FORM_EXACT, FORM_BLOCKED = 0, 1, 2
LAYOUT_BATCHED, LAYOUT_PUSH, LAYOUT_BLOCKED = 1, 2, 4
KDAMP = np.float32(0.85)  # include/common.h:18
EPSILON = 0.001           # src/pr/pr.h:4
MAX_ITER = 30             # src/pr/pr.h:5


class GprError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"gpr status {status}: {msg}")
        self.status = status


class PrOptions(C.Structure):
    _fields_ = [("damping", C.c_float), ("tol", C.c_double), ("max_iter", C.c_int),
                ("precision", C.c_int), ("loop", C.c_int), ("timeout_s", C.c_double),
                ("refine_max", C.c_int), ("variant", C.c_int), ("reserved", C.c_int * 1),
                ("form", C.c_int), ("ppr_repack", C.c_int), ("pad", C.c_int * 4)]


class LayoutOptions(C.Structure):
    _fields_ = [("sell_max", C.c_int), ("chunk", C.c_int), ("chunk_min", C.c_int),
                ("hot_entries", C.c_int), ("flags", C.c_int), ("block_rows", C.c_int),
                ("tile_words", C.c_int), ("blocked_long", C.c_int)]


class PrStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refine_iterations", C.c_int),
                ("residual", C.c_double), ("solve_ms", C.c_double),
                ("loop_ms", C.c_double), ("gpu_launches", C.c_int), ("reserved", C.c_int * 5)]

    def as_dict(self):
        return {"iterations": self.iterations, "refine_iterations": self.refine_iterations,
                "residual": self.residual, "solve_ms": self.solve_ms, "loop_ms": self.loop_ms,
                "gpu_launches": self.gpu_launches}


class TuneResult(C.Structure):
    _fields_ = [("layout", LayoutOptions), ("variant", C.c_int), ("from_cache", C.c_int),
                ("candidates", C.c_int), ("ms_per_sweep", C.c_double),
                ("default_ms_per_sweep", C.c_double), ("signature", C.c_char * 48)]

    def as_dict(self):
        lo = self.layout
        return {"sell_max": lo.sell_max, "chunk": lo.chunk, "chunk_min": lo.chunk_min,
                "hot_entries": lo.hot_entries, "blocked": bool(lo.flags & LAYOUT_BLOCKED),
                "block_rows": lo.block_rows, "tile_words": lo.tile_words,
                "blocked_long": lo.blocked_long, "variant": self.variant,
                "from_cache": bool(self.from_cache), "candidates": self.candidates,
                "ms_per_sweep": self.ms_per_sweep,
                "default_ms_per_sweep": self.default_ms_per_sweep,
                "signature": self.signature.decode()}


_LIB = None
_vp = C.c_void_p


def lib():
    """Load libgpr.so (built in-tree by ``build()``); raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run gardenia_ocl_b200.build() "
                           "(the CUDA library is required; there is no CPU path)")
    L = C.CDLL(LIB_PATH)
    I, LL, D, F = C.c_int, C.c_longlong, C.c_double, C.c_float
    sig = {
        "gpr_last_error": (C.c_char_p, []),
        "gpr_version": (C.c_char_p, []),
        "gpr_pr_opts_default": (I, [C.POINTER(PrOptions)]),
        "gpr_graph_create": (I, [I, LL, _vp, _vp, _vp, C.POINTER(_vp)]),
        "gpr_graph_create_ex": (I, [I, LL, _vp, _vp, _vp, C.POINTER(LayoutOptions),
                                    C.POINTER(_vp)]),
        "gpr_graph_destroy": (I, [_vp]),
        "gpr_graph_info": (I, [_vp, C.POINTER(I), C.POINTER(LL), C.POINTER(LL)]),
        "gpr_graph_layout": (I, [_vp, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(I),
                                 C.POINTER(LL), C.POINTER(LL)]),
        "gpr_graph_set_stream": (I, [_vp, _vp]),
        "gpr_graph_residuals": (I, [_vp, C.POINTER(D), I]),
        "gpr_pagerank": (I, [_vp, _vp, C.POINTER(PrOptions), C.POINTER(PrStats)]),
        "gpr_pr_residual_f64": (I, [_vp, _vp, F, C.POINTER(D)]),
        "gpr_pr_solver": (I, [I, I, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(PrOptions),
                              C.POINTER(PrStats)]),
        "gpr_page_rank": (I, [I, I, _vp, _vp, _vp, _vp, C.POINTER(PrOptions),
                              C.POINTER(PrStats)]),
        "gpr_pagerank_push": (I, [_vp, _vp, C.POINTER(PrOptions), C.POINTER(PrStats)]),
        "gpr_symgs_create": (I, [I, LL, _vp, _vp, _vp, _vp, _vp, I, C.POINTER(_vp)]),
        "gpr_symgs_destroy": (I, [_vp]),
        "gpr_symgs_apply": (I, [_vp, _vp, _vp, I, C.POINTER(D)]),
        "gpr_symgs_solver": (I, [I, I, _vp, _vp, _vp, _vp, _vp, _vp, _vp, I]),
        "gpr_ppr": (I, [_vp, I, _vp, _vp, C.POINTER(PrOptions), _vp, C.POINTER(PrStats)]),
        "gpr_pagerank_noalloc": (I, [I, I, _vp, _vp, _vp, _vp, C.POINTER(PrOptions),
                                     C.POINTER(PrStats), _vp]),
        "gpr_pagerank_noalloc_max_vertices": (LL, []),
        "gpr_matrix_create": (I, [I, LL, _vp, _vp, _vp, C.POINTER(_vp)]),
        "gpr_matrix_destroy": (I, [_vp]),
        "gpr_matrix_layout": (I, [_vp, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(LL)]),
        "gpr_spmv": (I, [_vp, _vp, _vp, _vp]),
        "gpr_spmv_solver": (I, [I, I, _vp, _vp, _vp, _vp, _vp]),
        "gpr_gen_rmat": (I, [I, I, D, D, D, C.c_ulonglong, I, C.POINTER(_vp), C.POINTER(_vp),
                             C.POINTER(_vp), C.POINTER(LL)]),
        "gpr_gen_stencil27": (I, [I, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                                  C.POINTER(LL)]),
        "gpr_gen_multigraph": (I, [I, I, I, I, I, D, C.c_ulonglong, _vp, C.POINTER(_vp),
                                   C.POINTER(_vp), C.POINTER(_vp), C.POINTER(LL)]),
        "gpr_multigraph_create": (I, [I, _vp, LL, _vp, _vp, _vp, C.POINTER(LayoutOptions),
                                      C.POINTER(_vp)]),
        "gpr_multigraph_destroy": (I, [_vp]),
        "gpr_multigraph_info": (I, [_vp, C.POINTER(I), C.POINTER(I), C.POINTER(LL),
                                    C.POINTER(I), C.POINTER(LL)]),
        "gpr_multigraph_set_stream": (I, [_vp, _vp]),
        "gpr_multigraph_pagerank": (I, [_vp, _vp, C.POINTER(PrOptions), _vp, _vp,
                                        C.POINTER(PrStats)]),
        "gpr_gen_uniform": (I, [LL, C.c_ulonglong, _vp]),
        "gpr_free": (I, [_vp]),
        "gpr_release_cached": (I, [C.POINTER(LL)]),
        "gpr_cached_bytes": (I, [C.POINTER(LL)]),
        "gpr_malloc": (I, [C.POINTER(_vp), C.c_size_t]),
        "gpr_memcpy": (I, [_vp, _vp, C.c_size_t]),
        "gpr_synchronize": (I, []),
        "gpr_set_device": (I, [I]),
        "gpr_read_graph": (I, [C.c_char_p, I, I, I, I, I, C.POINTER(I), C.POINTER(I),
                               C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
        "gpr_read_graph_free": (None, [_vp]),
        "gpr_csr_from_edges": (I, [I, LL, _vp, _vp, _vp, I, I, I, C.POINTER(_vp),
                                   C.POINTER(_vp), C.POINTER(_vp), C.POINTER(LL)]),
        "gpr_read_graph_gpu": (I, [C.c_char_p, I, I, I, I, I, C.POINTER(I), C.POINTER(LL),
                                   C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                                   C.POINTER(_vp)]),
        "gpr_read_graph_pr": (I, [C.c_char_p, I, C.POINTER(I), C.POINTER(LL), C.POINTER(LL),
                                  C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                                  C.POINTER(_vp), C.POINTER(_vp)]),
        "gpr_parse_edges": (I, [C.c_char_p, I, I, I, C.POINTER(I), C.POINTER(I), C.POINTER(LL),
                                C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
        "gpr_tune_graph": (I, [I, LL, _vp, _vp, _vp, C.c_char_p, I, C.POINTER(TuneResult)]),
        "gpr_tune_multigraph": (I, [I, _vp, LL, _vp, _vp, _vp, C.c_char_p, I,
                                    C.POINTER(LayoutOptions), C.POINTER(TuneResult)]),
        "gpr_tune_signature": (I, [I, LL, _vp, I, C.c_char_p, I]),
        "gpr_tune_cache_lookup": (I, [C.c_char_p, C.c_char_p, C.POINTER(TuneResult)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def build(verbose: bool = False) -> None:
    """Compile libgpr.so for sm_100a in-tree (make in csrc/)."""
    import subprocess
    subprocess.run(["make", "-s" if not verbose else "-j8", "-j8", "-C",
                    os.path.join(_HERE, "csrc")], check=True)
    global _LIB
    _LIB = None


def _check(status):
    if status != GPR_OK:
        msg = lib().gpr_last_error()
        raise GprError(status, msg.decode() if msg else "")


def _ptr(a, dtype=None):
    """Pointer to host numpy / device (data_ptr) memory; keeps numpy alive via the caller."""
    if a is None:
        return None, None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr()), a
    if isinstance(a, DeviceArray):
        return C.c_void_p(a.ptr), a
    arr = np.ascontiguousarray(a, dtype=dtype) if dtype is not None else np.ascontiguousarray(a)
    return C.c_void_p(arr.ctypes.data), arr


def options(tol=EPSILON, max_iter=MAX_ITER, damping=KDAMP, precision=PREC_FP32,
            loop=LOOP_AUTO, timeout_s=5.0, refine_max=64, variant=0, form=FORM_AUTO,
            ppr_repack=True) -> PrOptions:
    o = PrOptions()
    _check(lib().gpr_pr_opts_default(C.byref(o)))
    o.tol, o.max_iter, o.damping = float(tol), int(max_iter), float(damping)
    o.precision, o.loop, o.timeout_s, o.refine_max = int(precision), int(loop), float(timeout_s), int(refine_max)
    o.variant, o.form, o.ppr_repack = int(variant), int(form), 1 if ppr_repack else 0
    return o


class DeviceArray:
    """Device memory owned by libgpr (from the generators); freed on close()."""

    def __init__(self, ptr, n, dtype):
        self.ptr, self.n, self.dtype = int(ptr or 0), int(n), np.dtype(dtype)

    @property
    def nbytes(self):
        return self.n * self.dtype.itemsize

    def __len__(self):
        return self.n

    def data_ptr(self):
        return self.ptr

    def to_numpy(self):
        out = np.empty(self.n, dtype=self.dtype)
        if self.n:
            _check(lib().gpr_memcpy(C.c_void_p(out.ctypes.data), C.c_void_p(self.ptr), self.nbytes))
        return out

    def close(self):
        if self.ptr:
            lib().gpr_free(C.c_void_p(self.ptr))
            self.ptr = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# PageRank
# ---------------------------------------------------------------------------
class Graph:
    """Device-resident pull graph: in-CSR (row v = sources of edges u->v) plus
    the out-degree of every vertex (src/pr/omp_base.cc:9 arguments)."""

    def __init__(self, rowptr, col, outdeg, m=None, nnz=None, sell_max=0, chunk=0, chunk_min=0,
                 hot_entries=0, batched=False, push=False, blocked=False, block_rows=0,
                 tile_words=0, blocked_long=0):
        L = lib()
        m = int(len(rowptr) - 1) if m is None else int(m)
        nnz = int(len(col)) if nnz is None else int(nnz)
        pr, k0 = _ptr(rowptr, np.int32)
        pc, k1 = _ptr(col, np.int32)
        pd, k2 = _ptr(outdeg, np.int32)
        h = C.c_void_p()
        lo = LayoutOptions(int(sell_max), int(chunk), int(chunk_min), int(hot_entries),
                           (LAYOUT_BATCHED if batched else 0) | (LAYOUT_PUSH if push else 0) |
                           (LAYOUT_BLOCKED if blocked else 0), int(block_rows), int(tile_words),
                           int(blocked_long))
        _check(L.gpr_graph_create_ex(m, nnz, pr, pc, pd, C.byref(lo), C.byref(h)))
        self._h, self.m, self.nnz = h, m, nnz
        self.last_stats = None

    def pagerank(self, scores=None, opts: PrOptions | None = None, **kw):
        """Solve in place.  ``scores``: host numpy float32 (returned as a new
        array when None: uniform 1/m) or device memory (updated in place)."""
        o = opts if opts is not None else options(**kw)
        if scores is None:
            scores = np.full(self.m, np.float32(1.0) / np.float32(self.m), dtype=np.float32)
        if isinstance(scores, np.ndarray):
            if scores.dtype != np.float32 or not scores.flags.c_contiguous:
                raise TypeError("scores must be a contiguous float32 array")
        ps, keep = _ptr(scores)
        st = PrStats()
        _check(lib().gpr_pagerank(self._h, ps, C.byref(o), C.byref(st)))
        self.last_stats = st
        return scores, st

    def pagerank_push(self, scores=None, opts: PrOptions | None = None, **kw):
        """Push-style solve (graph created with push=True or batched=True);
        same arguments and results as ``pagerank``."""
        o = opts if opts is not None else options(**kw)
        if scores is None:
            scores = np.full(self.m, np.float32(1.0) / np.float32(self.m), dtype=np.float32)
        ps, keep = _ptr(scores)
        st = PrStats()
        _check(lib().gpr_pagerank_push(self._h, ps, C.byref(o), C.byref(st)))
        self.last_stats = st
        return scores, st

    def ppr(self, seeds, out=None, opts: PrOptions | None = None, **kw):
        """Batched personalized PageRank for len(seeds) <= 128 seed vertices
        (graph created with batched=True).  Returns (x[m, k] float32, iters[k],
        stats); ``out`` may be a device buffer of m*k floats."""
        o = opts if opts is not None else options(**kw)
        seeds = np.ascontiguousarray(seeds, dtype=np.int32)
        k = len(seeds)
        x = np.empty((self.m, k), dtype=np.float32) if out is None else out
        iters = np.zeros(k, dtype=np.int32)
        st = PrStats()
        px, keep = _ptr(x)
        _check(lib().gpr_ppr(self._h, k, C.c_void_p(seeds.ctypes.data), px, C.byref(o),
                             C.c_void_p(iters.ctypes.data), C.byref(st)))
        return x, iters, st

    def residuals(self):
        n = self.last_stats.iterations if self.last_stats else 0
        out = (C.c_double * max(n, 1))()
        _check(lib().gpr_graph_residuals(self._h, out, n))
        return np.array(out[:n])

    def residual_f64(self, scores, damping=KDAMP) -> float:
        ps, keep = _ptr(scores, np.float32)
        r = C.c_double()
        _check(lib().gpr_pr_residual_f64(self._h, ps, float(damping), C.byref(r)))
        return float(r.value)

    def layout(self):
        v = [C.c_int() for _ in range(4)] + [C.c_longlong() for _ in range(2)]
        _check(lib().gpr_graph_layout(self._h, *[C.byref(x) for x in v]))
        keys = ["n_long", "n_nz", "n_chunks", "n_slices", "long_elems", "sell_elems"]
        return {k: x.value for k, x in zip(keys, v)}

    def info(self):
        m, nnz, nb = C.c_int(), C.c_longlong(), C.c_longlong()
        _check(lib().gpr_graph_info(self._h, C.byref(m), C.byref(nnz), C.byref(nb)))
        return {"m": m.value, "nnz": nnz.value, "device_bytes": nb.value}

    def set_stream(self, stream_handle: int):
        _check(lib().gpr_graph_set_stream(self._h, C.c_void_p(stream_handle)))

    def close(self):
        if getattr(self, "_h", None):
            lib().gpr_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class MultiGraph:
    """Uneven batch of independent pull graphs stored as one block-diagonal
    graph: graph g owns vertices [voff[g], voff[g+1]) and the in-edges of its
    rows come from that range (global vertex ids).  ``layouts``: None, or one
    dict per graph with any of sell_max / chunk / chunk_min (each graph's own
    bins) and blocked / block_rows / tile_words (the blocked form for the
    whole batch, as ``tune_multigraph`` returns them).  Every graph is solved as ``Graph.pagerank`` solves it alone, all
    in one persistent launch.  ``blocked``: also build the blocked form's
    layout (each graph's rows in blocks; ``block_rows`` / ``tile_words`` as
    for ``Graph``), which ``pagerank`` uses from 50.3M edges up (AUTO) or when
    asked with ``form=FORM_BLOCKED``."""

    def __init__(self, rowptr, col, outdeg, voff, nnz=None, layouts=None, blocked=False,
                 block_rows=0, tile_words=0):
        L = lib()
        self.voff = np.ascontiguousarray(voff, dtype=np.int32)
        self.n_graphs = len(self.voff) - 1
        self.m = int(self.voff[-1])
        nnz = int(len(col)) if nnz is None else int(nnz)
        lo = None
        if layouts is not None or blocked:
            if layouts is not None and len(layouts) != self.n_graphs:
                raise ValueError("one layout per graph")
            lo = (LayoutOptions * self.n_graphs)()
            for i in range(self.n_graphs):
                d = (layouts[i] if layouts is not None else None) or {}
                b = blocked or bool(d.get("blocked", False))
                lo[i] = LayoutOptions(int(d.get("sell_max", 0)), int(d.get("chunk", 0)),
                                      int(d.get("chunk_min", 0)), 0,
                                      LAYOUT_BLOCKED if b else 0,
                                      int(block_rows or d.get("block_rows", 0)),
                                      int(tile_words or d.get("tile_words", 0)), 0)
        pr, k0 = _ptr(rowptr, np.int32)
        pc, k1 = _ptr(col, np.int32)
        pd, k2 = _ptr(outdeg, np.int32)
        h = C.c_void_p()
        _check(L.gpr_multigraph_create(self.n_graphs, C.c_void_p(self.voff.ctypes.data), nnz,
                                       pr, pc, pd, lo, C.byref(h)))
        self._h, self.nnz = h, nnz
        self.last_stats = None

    def initial_scores(self):
        """1/m_g on every vertex of graph g (src/pr/main.cc:27-28, per graph)."""
        sizes = np.diff(self.voff)
        vals = np.where(sizes > 0, np.float32(1.0) / np.maximum(sizes, 1).astype(np.float32),
                        np.float32(0.0)).astype(np.float32)
        return np.repeat(vals, sizes)

    def pagerank(self, scores=None, opts: PrOptions | None = None, **kw):
        """Returns (scores, iters[n_graphs], residuals[n_graphs], stats);
        ``scores`` host float32 (new array of 1/m_g when None) or device
        memory updated in place."""
        o = opts if opts is not None else options(**kw)
        if scores is None:
            scores = self.initial_scores()
        if isinstance(scores, np.ndarray) and (scores.dtype != np.float32 or
                                               not scores.flags.c_contiguous):
            raise TypeError("scores must be a contiguous float32 array")
        iters = np.zeros(self.n_graphs, dtype=np.int32)
        res = np.zeros(self.n_graphs, dtype=np.float64)
        ps, keep = _ptr(scores)
        st = PrStats()
        _check(lib().gpr_multigraph_pagerank(self._h, ps, C.byref(o),
                                             C.c_void_p(iters.ctypes.data),
                                             C.c_void_p(res.ctypes.data), C.byref(st)))
        self.last_stats = st
        return scores, iters, res, st

    def info(self):
        g, m, nnz, u, es = C.c_int(), C.c_int(), C.c_longlong(), C.c_int(), C.c_longlong()
        _check(lib().gpr_multigraph_info(self._h, C.byref(g), C.byref(m), C.byref(nnz),
                                         C.byref(u), C.byref(es)))
        return {"n_graphs": g.value, "m": m.value, "nnz": nnz.value, "units": u.value,
                "edge_slots": es.value}

    def set_stream(self, stream_handle: int):
        _check(lib().gpr_multigraph_set_stream(self._h, C.c_void_p(stream_handle)))

    def close(self):
        if getattr(self, "_h", None):
            lib().gpr_multigraph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def PRSolver(m, nnz, in_row_offsets, in_column_indices, out_row_offsets, out_column_indices,
             degree, scores, tol=EPSILON, max_iter=MAX_ITER, **kw):
    """src/pr/pr.h:23.  ``scores`` (float32, host or device) is updated in
    place; returns the stats (iterations = sweeps executed)."""
    o = options(tol=tol, max_iter=max_iter, **kw)
    st = PrStats()
    ptrs = [_ptr(a, np.int32) for a in (in_row_offsets, in_column_indices, out_row_offsets,
                                        out_column_indices, degree)]
    ps, keep = _ptr(scores)
    if isinstance(scores, np.ndarray) and scores.dtype != np.float32:
        raise TypeError("scores must be float32")
    _check(lib().gpr_pr_solver(int(m), int(nnz), *[p for p, _ in ptrs], ps, C.byref(o), C.byref(st)))
    return st


def PageRank(m, nnz, row_offsets, column_indices, degree, scores, tol=EPSILON,
             max_iter=MAX_ITER, **kw):
    """Pull PageRank over the in-CSR and out-degree; ``scores`` updated in place."""
    o = options(tol=tol, max_iter=max_iter, **kw)
    st = PrStats()
    ptrs = [_ptr(a, np.int32) for a in (row_offsets, column_indices, degree)]
    ps, keep = _ptr(scores)
    if isinstance(scores, np.ndarray) and scores.dtype != np.float32:
        raise TypeError("scores must be float32")
    _check(lib().gpr_page_rank(int(m), int(nnz), *[p for p, _ in ptrs], ps, C.byref(o), C.byref(st)))
    return st


def pagerank_noalloc(m, nnz, d_rowptr, d_col, d_outdeg, d_scores, stream_handle=0,
                     tol=EPSILON, max_iter=MAX_ITER, **kw):
    """PageRank that allocates no device memory (gpr_pagerank_noalloc): every
    array must already be on the device; ``d_scores`` is updated in place.
    For callers whose device memory belongs to their own allocator."""
    o = options(tol=tol, max_iter=max_iter, **kw)
    st = PrStats()
    _check(lib().gpr_pagerank_noalloc(int(m), int(nnz), _ptr(d_rowptr)[0], _ptr(d_col)[0],
                                      _ptr(d_outdeg)[0], _ptr(d_scores)[0], C.byref(o),
                                      C.byref(st), C.c_void_p(stream_handle)))
    return st


def pagerank_noalloc_max_vertices() -> int:
    return int(lib().gpr_pagerank_noalloc_max_vertices())


# ---------------------------------------------------------------------------
# SpMV
# ---------------------------------------------------------------------------
class Matrix:
    """Device-resident CSR matrix for y <- y + A x."""

    def __init__(self, Ap, Aj, Ax, m=None, nnz=None):
        m = int(len(Ap) - 1) if m is None else int(m)
        nnz = int(len(Aj)) if nnz is None else int(nnz)
        pa, k0 = _ptr(Ap, np.int32)
        pj, k1 = _ptr(Aj, np.int32)
        px, k2 = _ptr(Ax, np.float32)
        h = C.c_void_p()
        _check(lib().gpr_matrix_create(m, nnz, pa, pj, px, C.byref(h)))
        self._h, self.m, self.nnz = h, m, nnz

    def spmv(self, d_x, d_y, stream_handle: int = 0):
        """Device x, y (data_ptr objects); asynchronous on the stream."""
        _check(lib().gpr_spmv(self._h, _ptr(d_x)[0], _ptr(d_y)[0], C.c_void_p(stream_handle)))

    def layout(self):
        v = [C.c_int() for _ in range(3)] + [C.c_longlong()]
        _check(lib().gpr_matrix_layout(self._h, *[C.byref(x) for x in v]))
        return dict(zip(["n_long", "n_chunks", "n_slices", "sell_elems"], [x.value for x in v]))

    def close(self):
        if getattr(self, "_h", None):
            lib().gpr_matrix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SymGS:
    """Multicolour symmetric Gauss-Seidel smoother (src/symgs): the matrix
    laid out per colour on the device; ``apply`` runs sweeps in place."""

    def __init__(self, Ap, Aj, Ax, indices, color_offsets, m=None, nnz=None):
        m = int(len(Ap) - 1) if m is None else int(m)
        nnz = int(len(Aj)) if nnz is None else int(nnz)
        co = np.ascontiguousarray(color_offsets, dtype=np.int32)
        args = [_ptr(Ap, np.int32), _ptr(Aj, np.int32), _ptr(Ax, np.float32),
                _ptr(indices, np.int32)]
        h = C.c_void_p()
        _check(lib().gpr_symgs_create(m, nnz, *[p for p, _ in args], C.c_void_p(co.ctypes.data),
                                      len(co) - 1, C.byref(h)))
        self._h, self.m = h, m

    def apply(self, x, b, sweeps=1):
        """x (float32 host array or device memory) updated in place; returns
        the device time of the launch in ms."""
        px, k0 = _ptr(x)
        pb, k1 = _ptr(b, np.float32)
        ms = C.c_double()
        _check(lib().gpr_symgs_apply(self._h, px, pb, int(sweeps), C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "_h", None):
            lib().gpr_symgs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def SymGSSolver(m, nnz, Ap, Aj, indices, Ax, x, b, color_offsets):
    """src/symgs/symgs.h:28: one sweep, ``x`` (float32 numpy) updated in place."""
    if not (isinstance(x, np.ndarray) and x.dtype == np.float32 and x.flags.c_contiguous):
        raise TypeError("x must be a contiguous float32 numpy array")
    co = np.ascontiguousarray(color_offsets, dtype=np.int32)
    args = [_ptr(Ap, np.int32), _ptr(Aj, np.int32), _ptr(indices, np.int32),
            _ptr(Ax, np.float32)]
    pb, kb = _ptr(b, np.float32)
    _check(lib().gpr_symgs_solver(int(m), int(nnz), *[p for p, _ in args],
                                  C.c_void_p(x.ctypes.data), pb, C.c_void_p(co.ctypes.data),
                                  len(co) - 1))


def SpmvSolver(m, nnz, Ap, Aj, Ax, x, y):
    """src/spmv/spmv.h:29: y <- y + A x, ``y`` (float32 numpy) updated in place."""
    if not (isinstance(y, np.ndarray) and y.dtype == np.float32 and y.flags.c_contiguous):
        raise TypeError("y must be a contiguous float32 numpy array")
    args = [_ptr(Ap, np.int32), _ptr(Aj, np.int32), _ptr(Ax, np.float32), _ptr(x, np.float32)]
    _check(lib().gpr_spmv_solver(int(m), int(nnz), *[p for p, _ in args],
                                 C.c_void_p(y.ctypes.data)))


# ---------------------------------------------------------------------------
# Inputs: loaders and generators
# ---------------------------------------------------------------------------
def read_graph(path, symmetrize=False, transpose=False, sorted=True, remove_selfloops=True,
               remove_redundents=True):
    """include/graph_io.h:280 with the same flags.  Returns
    (m, nnz, row_offsets, column_indices, degree, weight) as numpy arrays."""
    L = lib()
    m, nnz = C.c_int(), C.c_int()
    p = [C.c_void_p() for _ in range(4)]
    _check(L.gpr_read_graph(os.fsencode(path), int(symmetrize), int(transpose), int(sorted),
                            int(remove_selfloops), int(remove_redundents), C.byref(m),
                            C.byref(nnz), *[C.byref(q) for q in p]))
    mm, nz = m.value, nnz.value

    def take(ptr, n, ct, dt):
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(max(n, 1),))[:n].astype(dt, copy=True)
        L.gpr_read_graph_free(ptr)
        return a
    rp = take(p[0], mm + 1, C.c_int, np.int32)
    col = take(p[1], nz, C.c_int, np.int32)
    deg = take(p[2], mm, C.c_int, np.int32)
    wt = take(p[3], nz, C.c_float, np.float32)
    return mm, nz, rp, col, deg, wt


def parse_edges(path, symmetrize=False, transpose=False, threads=0):
    """The file's edges as the reference pushes them into per-vertex lists
    (multithreaded parse, gpr_parse_edges): returns (m, nnz_header, row, col,
    weight) numpy arrays in push order."""
    L = lib()
    m, nnz, n = C.c_int(), C.c_int(), C.c_longlong()
    p = [C.c_void_p() for _ in range(3)]
    st = L.gpr_parse_edges(os.fsencode(path), int(symmetrize), int(transpose), int(threads),
                           C.byref(m), C.byref(nnz), C.byref(n), *[C.byref(q) for q in p])
    _check(st)
    k = n.value

    def take(ptr, ct, dt):
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(max(k, 1),))[:k].astype(dt, copy=True)
        L.gpr_read_graph_free(ptr)
        return a
    return (m.value, nnz.value, take(p[0], C.c_int, np.int32), take(p[1], C.c_int, np.int32),
            take(p[2], C.c_float, np.float32))


class DeviceCSR:
    """CSR arrays in device memory produced by a generator."""

    def __init__(self, m, nnz, rowptr, col, third, third_dtype):
        self.m, self.nnz = m, nnz
        self.rowptr = DeviceArray(rowptr, m + 1, np.int32)
        self.col = DeviceArray(col, nnz, np.int32)
        self.third = DeviceArray(third, m if third_dtype == np.int32 else nnz, third_dtype) \
            if third else None

    def close(self):
        for a in (self.rowptr, self.col, self.third):
            if a is not None:
                a.close()


def csr_from_edges(m, row, col, wt=None, sorted=True, remove_selfloops=True,
                   remove_redundents=True):
    """fill_data on the GPU over a push list (gpr_csr_from_edges): returns
    (DeviceCSR with third = weights or None)."""
    pr, k0 = _ptr(row, np.int32)
    pc, k1 = _ptr(col, np.int32)
    pw, k2 = _ptr(wt, np.float32) if wt is not None else (None, None)
    rp, cp, wp, nnz = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_longlong()
    _check(lib().gpr_csr_from_edges(int(m), int(len(row)), pr, pc, pw, int(sorted),
                                    int(remove_selfloops), int(remove_redundents), C.byref(rp),
                                    C.byref(cp), C.byref(wp) if wt is not None else None,
                                    C.byref(nnz)))
    return DeviceCSR(int(m), nnz.value, rp.value, cp.value,
                     wp.value if wt is not None else None, np.float32)


def read_graph_gpu(path, symmetrize=False, transpose=False, sorted=True, remove_selfloops=True,
                   remove_redundents=True):
    """read_graph with a multithreaded parse and the CSR built on the GPU:
    returns (DeviceCSR with third = degree, weights DeviceArray)."""
    m, nnz = C.c_int(), C.c_longlong()
    rp, cp, dp, wp = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(lib().gpr_read_graph_gpu(os.fsencode(path), int(symmetrize), int(transpose),
                                    int(sorted), int(remove_selfloops), int(remove_redundents),
                                    C.byref(m), C.byref(nnz), C.byref(rp), C.byref(cp),
                                    C.byref(dp), C.byref(wp)))
    return (DeviceCSR(m.value, nnz.value, rp.value, cp.value, dp.value, np.int32),
            DeviceArray(wp.value, nnz.value, np.float32))


def read_graph_pr(path, symmetrize=False):
    """The PR driver's two reads (src/pr/main.cc:23-24) from one parse:
    returns (out DeviceCSR with third = out-degree, in DeviceCSR with third =
    out-degree as well -- the PRSolver arguments)."""
    m, no, ni = C.c_int(), C.c_longlong(), C.c_longlong()
    p = [C.c_void_p() for _ in range(5)]
    _check(lib().gpr_read_graph_pr(os.fsencode(path), int(symmetrize), C.byref(m), C.byref(no),
                                   C.byref(ni), *[C.byref(q) for q in p]))
    out = DeviceCSR(m.value, no.value, p[0].value, p[1].value, p[2].value, np.int32)
    inn = DeviceCSR(m.value, ni.value, p[3].value, p[4].value, None, np.int32)
    return out, inn


def gen_rmat(scale, edge_factor=16, seed=1, abc=(0.57, 0.19, 0.19), scramble=True) -> DeviceCSR:
    """Seeded RMAT pull graph on the GPU: rowptr, col (in-CSR), third = out-degree."""
    rp, cp, dp, nnz = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_longlong()
    _check(lib().gpr_gen_rmat(int(scale), int(edge_factor), abc[0], abc[1], abc[2], int(seed),
                              1 if scramble else 0, C.byref(rp), C.byref(cp), C.byref(dp),
                              C.byref(nnz)))
    return DeviceCSR(1 << scale, nnz.value, rp.value, cp.value, dp.value, np.int32)


def gen_stencil27(n) -> DeviceCSR:
    """27-point Laplacian on an n^3 grid on the GPU: rowptr, col, third = values."""
    ap, aj, ax, nnz = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_longlong()
    _check(lib().gpr_gen_stencil27(int(n), C.byref(ap), C.byref(aj), C.byref(ax), C.byref(nnz)))
    return DeviceCSR(n ** 3, nnz.value, ap.value, aj.value, ax.value, np.float32)


def gen_multigraph(n_graphs, m_min=1000, m_max=500000, seed=1, er_deg=8, cl_deg=16,
                   gamma=2.1):
    """Seeded uneven batch on the GPU (gpr_gen_multigraph): returns
    (DeviceCSR with third = out-degree, voff[n_graphs + 1] numpy)."""
    voff = np.zeros(n_graphs + 1, dtype=np.int32)
    rp, cp, dp, nnz = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_longlong()
    _check(lib().gpr_gen_multigraph(int(n_graphs), int(m_min), int(m_max), int(er_deg),
                                    int(cl_deg), float(gamma), int(seed),
                                    C.c_void_p(voff.ctypes.data), C.byref(rp), C.byref(cp),
                                    C.byref(dp), C.byref(nnz)))
    return DeviceCSR(int(voff[-1]), nnz.value, rp.value, cp.value, dp.value, np.int32), voff


def gen_uniform(n, seed, d_out) -> None:
    _check(lib().gpr_gen_uniform(int(n), int(seed), _ptr(d_out)[0]))


# ---------------------------------------------------------------------------
# Autotuner
# ---------------------------------------------------------------------------
def tune_graph(rowptr, col, outdeg, m=None, nnz=None, cache=None, sweeps=5) -> dict:
    """Layout (exact order or blocked, bins, hot prefix) and kernel variant for
    this graph's in-degree distribution (gpr_tune_graph).  Pass the layout
    keys (sell_max, chunk, chunk_min, hot_entries, blocked, block_rows,
    tile_words, blocked_long) to ``Graph(...)`` and ``variant`` to ``pagerank``; ``cache``:
    path of the text cache (or None)."""
    m = int(len(rowptr) - 1) if m is None else int(m)
    nnz = int(len(col)) if nnz is None else int(nnz)
    pr, k0 = _ptr(rowptr, np.int32)
    pc, k1 = _ptr(col, np.int32)
    pd, k2 = _ptr(outdeg, np.int32)
    r = TuneResult()
    _check(lib().gpr_tune_graph(m, nnz, pr, pc, pd, os.fsencode(cache) if cache else None,
                                int(sweeps), C.byref(r)))
    return r.as_dict()


def tune_multigraph(rowptr, col, outdeg, voff, nnz=None, cache=None, sweeps=5):
    """Per-graph bins, or the blocked form, for a batch (gpr_tune_multigraph):
    returns (layouts, summary), ``layouts`` ready for
    ``MultiGraph(..., layouts=layouts)``."""
    voff = np.ascontiguousarray(voff, dtype=np.int32)
    n = len(voff) - 1
    nnz = int(len(col)) if nnz is None else int(nnz)
    pr, k0 = _ptr(rowptr, np.int32)
    pc, k1 = _ptr(col, np.int32)
    pd, k2 = _ptr(outdeg, np.int32)
    lo = (LayoutOptions * n)()
    r = TuneResult()
    _check(lib().gpr_tune_multigraph(n, C.c_void_p(voff.ctypes.data), nnz, pr, pc, pd,
                                     os.fsencode(cache) if cache else None, int(sweeps), lo,
                                     C.byref(r)))
    layouts = [{"sell_max": x.sell_max, "chunk": x.chunk, "chunk_min": x.chunk_min,
                "blocked": bool(x.flags & LAYOUT_BLOCKED), "block_rows": x.block_rows,
                "tile_words": x.tile_words} for x in lo]
    return layouts, r.as_dict()


def tune_signature(rowptr, batch=False) -> str:
    """Distribution signature (the cache key) of a host row-offset array."""
    rp = np.ascontiguousarray(rowptr, dtype=np.int32)
    buf = C.create_string_buffer(64)
    _check(lib().gpr_tune_signature(len(rp) - 1, int(rp[-1] - rp[0]) if len(rp) else 0,
                                    C.c_void_p(rp.ctypes.data), 1 if batch else 0, buf, 64))
    return buf.value.decode()


def tune_cache_lookup(cache, signature):
    r = TuneResult()
    st = lib().gpr_tune_cache_lookup(os.fsencode(cache), signature.encode(), C.byref(r))
    return r.as_dict() if st == GPR_OK else None


def set_device(device: int):
    _check(lib().gpr_set_device(int(device)))


def release_cached() -> int:
    """Return the library's cached device blocks to the CUDA driver; returns bytes."""
    n = C.c_longlong()
    _check(lib().gpr_release_cached(C.byref(n)))
    return n.value


def cached_bytes() -> int:
    n = C.c_longlong()
    _check(lib().gpr_cached_bytes(C.byref(n)))
    return n.value


def synchronize():
    _check(lib().gpr_synchronize())


def version() -> str:
    return lib().gpr_version().decode()
