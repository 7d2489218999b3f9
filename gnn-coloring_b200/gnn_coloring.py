"""ctypes binding of libgnncolor.so (the B200 greedy-coloring library).

Two layers, mirroring include/:
  * the native device API (include/gnn_coloring.h): Context, Graph, Model, priority(), color();
  * the reference-named drop-in functions (include/coloring.h, first_fit.h, ... of
    KennethLangedal/GNN-COLORING), exposed as ``legacy.<name>`` with numpy arrays.

Plus seeded graph generators and .gnn model helpers (host side).

The library is the product; it runs only on the GPU.  Importing this module fails loudly if the
in-tree shared library is missing; creating a Context fails with GCError(GC_ERR_NODEV) when no
CUDA device is visible.  Nothing here falls back to the CPU.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import weakref
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgnncolor.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (or __graft_entry__.build())")
lib = C.CDLL(LIB_PATH)

u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p

STATUS = {
    0: "GC_OK", 1: "GC_ERR_INVALID", 2: "GC_ERR_NOMEM", 3: "GC_ERR_CUDA", 4: "GC_ERR_DEVICE",
    5: "GC_ERR_IO", 6: "GC_ERR_FORMAT", 7: "GC_ERR_BUDGET", 8: "GC_ERR_NODEV", 9: "GC_ERR_STATE",
}
GC_FF, GC_LF, GC_LLF, GC_SL, GC_SLL, GC_GNN = range(6)
HEURISTICS = {"FF": GC_FF, "LF": GC_LF, "LLF": GC_LLF, "SL": GC_SL, "SLL": GC_SLL, "GNN": GC_GNN}


class GCError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {msg}" if msg else self.name)


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


# native API
_sig("gc_status_string", C.c_char_p, C.c_int)
_sig("gc_ctx_create", C.c_int, C.c_int, C.POINTER(vp))
_sig("gc_ctx_destroy", None, vp)
_sig("gc_last_error", C.c_char_p, vp)
_sig("gc_ctx_stream", vp, vp)
_sig("gc_sync", C.c_int, vp)
_sig("gc_ctx_launches", C.c_uint64, vp)
_sig("gc_graph_upload", C.c_int, vp, C.c_uint32, u32p, u32p, C.POINTER(vp))
_sig("gc_graph_create", C.c_int, vp, C.c_uint32, C.c_uint32, C.POINTER(vp))
_sig("gc_graph_reupload", C.c_int, vp, vp, C.c_uint32, u32p, u32p)
_sig("gc_graph_wrap_device", C.c_int, vp, C.c_uint32, C.c_uint32, vp, vp, C.POINTER(vp))
_sig("gc_graph_free", None, vp)
_sig("gc_graph_num_vertices", C.c_uint32, vp)
_sig("gc_graph_num_edges", C.c_uint32, vp)
_sig("gc_graph_max_degree", C.c_uint32, vp)
_sig("gc_graph_device_keys", vp, vp)
_sig("gc_graph_device_colors", vp, vp)
_sig("gc_model_load", C.c_int, vp, C.c_char_p, C.POINTER(vp))
_sig("gc_model_create", C.c_int, vp, C.c_int, C.c_int, f32p, C.POINTER(vp))
_sig("gc_model_free", None, vp)
_sig("gc_model_layers", C.c_int, vp)
_sig("gc_priority", C.c_int, vp, vp, C.c_int, vp)
_sig("gc_priority_set", C.c_int, vp, vp, f64p)
_sig("gc_color", C.c_int, vp, vp, C.c_int, C.POINTER(C.c_int))
_sig("gc_recolor", C.c_int, vp, vp, C.c_int, C.POINTER(C.c_int))
_sig("gc_validate", C.c_int, vp, vp, C.POINTER(C.c_int))
_sig("gc_upload_colors", C.c_int, vp, vp, i32p)
_sig("gc_download_colors", C.c_int, vp, vp, i32p)
_sig("gc_download_priority", C.c_int, vp, vp, f64p)
# host helpers
_sig("gc_mtx_read", C.c_int, C.c_char_p, u32p, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_graph_load_mtx", C.c_int, vp, C.c_char_p, C.POINTER(vp))
_sig("gc_mtx_read_device", C.c_int, vp, C.c_char_p, u32p, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_mtx_write", C.c_int, C.c_char_p, C.c_uint32, u32p, u32p)
_sig("gc_csr_from_pairs", C.c_int, C.c_uint32, C.c_uint64, u32p, u32p, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_model_read", C.c_int, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(f32p))
_sig("gc_host_free", None, vp)
_sig("gc_gen_er", C.c_int, C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_gen_rmat", C.c_int, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
     C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_gen_rgg2d", C.c_int, C.c_uint32, C.c_double, C.c_uint64, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_gen_stencil27", C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_gen_mixed", C.c_int, C.c_uint64, C.c_uint32, C.c_uint32, u32p, C.POINTER(C.c_int), f64p,
     C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_gen_mixed_batch", C.c_int, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(u32p),
     C.POINTER(u32p), C.POINTER(u32p))


class Tuning(C.Structure):
    """gc_tuning: what the batch autotuner may change (never a color or priority bit)."""
    _fields_ = [("warp_degree", C.c_uint32), ("hub_degree", C.c_uint32), ("schedule", C.c_int),
                ("jp_ctas_per_sm", C.c_int), ("jp_tight", C.c_uint), ("jp_nap", C.c_uint),
                ("gnn_warp_degree", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


GC_SCHEDULE_DEGREE, GC_SCHEDULE_SEGMENT = 0, 1
SCHEDULES = {"degree": GC_SCHEDULE_DEGREE, "segment": GC_SCHEDULE_SEGMENT}

# batches
_sig("gc_batch_upload", C.c_int, vp, C.c_uint32, u32p, u32p, u32p, C.POINTER(vp))
_sig("gc_batch_upload_graphs", C.c_int, vp, C.c_uint32, u32p, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(vp))
_sig("gc_batch_create", C.c_int, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(vp))
_sig("gc_batch_reupload_graphs", C.c_int, vp, vp, C.c_uint32, u32p, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_batch_free", None, vp)
_sig("gc_batch_num_graphs", C.c_uint32, vp)
_sig("gc_batch_num_vertices", C.c_uint32, vp)
_sig("gc_batch_num_edges", C.c_uint32, vp)
_sig("gc_batch_device_bytes", C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int)
_sig("gc_batch_graph", vp, vp)
_sig("gc_batch_color", C.c_int, vp, vp, C.c_int, vp, C.c_int, i32p)
_sig("gc_batch_download_colors", C.c_int, vp, vp, i32p)
_sig("gc_batch_autotune", C.c_int, vp, vp, C.c_int, vp, C.c_int, C.c_int, C.POINTER(Tuning), f64p)
_sig("gc_batch_set_tuning", C.c_int, vp, vp, C.POINTER(Tuning))
_sig("gc_batch_get_tuning", C.c_int, vp, C.POINTER(Tuning))
_sig("gc_tuning_default", None, C.POINTER(Tuning))

_sig("gc_batch_reupload", C.c_int, vp, vp, C.c_uint32, u32p, u32p, u32p)
_sig("gc_batch_color_once", C.c_int, vp, vp, C.c_int, vp, C.c_int, i32p)


class ServeConfig(C.Structure):
    """gc_serve_config."""
    _fields_ = [("device", C.c_int), ("lanes", C.c_uint32), ("hbm_budget", C.c_uint64),
                ("slot_graphs", C.c_uint32), ("slot_vertices", C.c_uint32), ("slot_edges", C.c_uint32),
                ("batch_max_job_vertices", C.c_uint32)]


class JobInfo(C.Structure):
    """gc_job_info: outcome and timing of one served job."""
    _fields_ = [("status", C.c_int), ("colors", C.c_int), ("N", C.c_uint32), ("M", C.c_uint32),
                ("batch_jobs", C.c_uint32), ("lane", C.c_uint32), ("queue_ms", C.c_double),
                ("run_ms", C.c_double), ("latency_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeStats(C.Structure):
    """gc_serve_stats."""
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("rejected", C.c_uint64), ("edges", C.c_uint64), ("launches", C.c_uint64),
                ("batched_jobs", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("max_ms", C.c_double), ("span_s", C.c_double),
                ("edges_per_s", C.c_double), ("budget_bytes", C.c_uint64), ("reserved_bytes", C.c_uint64),
                ("peak_reserved_bytes", C.c_uint64), ("pool_peak_bytes", C.c_uint64), ("lanes", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_sig("gc_serve_config_default", None, C.POINTER(ServeConfig))
_sig("gc_serve_create", C.c_int, C.POINTER(ServeConfig), C.POINTER(vp))
_sig("gc_serve_add_model", C.c_int, vp, C.c_int, C.c_int, f32p)
_sig("gc_serve_submit", C.c_int, vp, C.c_uint32, u32p, u32p, C.c_int, C.c_int, C.c_int, i32p,
     C.POINTER(C.c_uint64))
_sig("gc_serve_test", C.c_int, vp, C.c_uint64, C.POINTER(C.c_int))
_sig("gc_serve_wait", C.c_int, vp, C.c_uint64, C.POINTER(JobInfo))
_sig("gc_serve_drain", C.c_int, vp)
_sig("gc_serve_replay", C.c_int, vp, C.c_uint32, f64p, u32p, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(C.c_int),
     C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(i32p), C.POINTER(JobInfo))
_sig("gc_serve_register", C.c_int, vp, C.c_uint32, u32p, u32p, C.POINTER(C.c_uint64))
_sig("gc_serve_unregister", C.c_int, vp, C.c_uint64)
_sig("gc_serve_submit_registered", C.c_int, vp, C.c_uint64, C.c_int, C.c_int, C.c_int, i32p, C.POINTER(C.c_uint64))
_sig("gc_serve_replay_registered", C.c_int, vp, C.c_uint32, f64p, C.POINTER(C.c_uint64), C.POINTER(C.c_int),
     C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(i32p), C.POINTER(JobInfo))
_sig("gc_batch_reupload_device_graphs", C.c_int, vp, vp, C.c_uint32, u32p, u32p, C.POINTER(u32p), C.POINTER(u32p))
_sig("gc_serve_read_stats", C.c_int, vp, C.POINTER(ServeStats))
_sig("gc_serve_reset_stats", None, vp)
_sig("gc_serve_last_error", C.c_char_p, vp)
_sig("gc_serve_destroy", None, vp)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _check(status: int, ctx_handle=None, what: str = ""):
    if status != 0:
        msg = what
        if ctx_handle:
            detail = lib.gc_last_error(ctx_handle)
            if detail:
                msg = f"{what}: {detail.decode()}" if what else detail.decode()
        raise GCError(status, msg)


# ---- host-side graphs ------------------------------------------------------------------------

def _take_csr(N: int, Vp, Ep) -> Tuple[int, np.ndarray, np.ndarray]:
    V = np.ctypeslib.as_array(Vp, shape=(N + 1,)).copy()
    M = int(V[N])
    E = np.ctypeslib.as_array(Ep, shape=(max(M, 1),))[:M].copy() if M else np.zeros(0, np.uint32)
    lib.gc_host_free(C.cast(Vp, vp))
    lib.gc_host_free(C.cast(Ep, vp))
    return N, V, E


def gen_er(n: int, m: int, seed: int):
    Vp, Ep = u32p(), u32p()
    _check(lib.gc_gen_er(n, m, seed, C.byref(Vp), C.byref(Ep)), what="gen_er")
    return _take_csr(n, Vp, Ep)


def gen_rmat(n: int, ef: float, seed: int, a: float = 0.57, b: float = 0.19, c: float = 0.19):
    Vp, Ep = u32p(), u32p()
    _check(lib.gc_gen_rmat(n, ef, a, b, c, seed, C.byref(Vp), C.byref(Ep)), what="gen_rmat")
    return _take_csr(n, Vp, Ep)


def gen_rgg2d(n: int, radius: float, seed: int):
    Vp, Ep = u32p(), u32p()
    _check(lib.gc_gen_rgg2d(n, radius, seed, C.byref(Vp), C.byref(Ep)), what="gen_rgg2d")
    return _take_csr(n, Vp, Ep)


def gen_stencil27(nx: int, ny: int, nz: int):
    Vp, Ep = u32p(), u32p()
    _check(lib.gc_gen_stencil27(nx, ny, nz, C.byref(Vp), C.byref(Ep)), what="gen_stencil27")
    return _take_csr(nx * ny * nz, Vp, Ep)


def csr_from_pairs(n: int, I: np.ndarray, J: np.ndarray):
    I = np.ascontiguousarray(I, dtype=np.uint32)
    J = np.ascontiguousarray(J, dtype=np.uint32)
    Vp, Ep = u32p(), u32p()
    _check(lib.gc_csr_from_pairs(n, len(I), _ptr(I, u32p), _ptr(J, u32p), C.byref(Vp), C.byref(Ep)),
           what="csr_from_pairs")
    return _take_csr(n, Vp, Ep)


def gen_mixed(seed: int, n_min: int = 1000, n_max: int = 200000):
    """One graph of a mixed batch (gc_gen_mixed): (N, V, E, kind, param), kind 0 = ER, 1 = R-MAT."""
    Vp, Ep = u32p(), u32p()
    n, kind, param = C.c_uint32(), C.c_int(), C.c_double()
    _check(lib.gc_gen_mixed(seed, n_min, n_max, C.byref(n), C.byref(kind), C.byref(param), C.byref(Vp), C.byref(Ep)),
           what="gen_mixed")
    N, V, E = _take_csr(n.value, Vp, Ep)
    return N, V, E, kind.value, param.value


def _owned(p, count: int) -> np.ndarray:
    """A uint32 array over a buffer the library malloc'd, freed when the array is collected (no copy:
    batches reach several GB)."""
    if count == 0:
        lib.gc_host_free(C.cast(p, vp))
        return np.zeros(0, np.uint32)
    a = np.ctypeslib.as_array(p, shape=(count,))
    weakref.finalize(a, lib.gc_host_free, C.cast(p, vp))
    return a


def gen_mixed_batch(G: int, seed0: int, n_min: int = 1000, n_max: int = 200000):
    """G mixed graphs as one segmented CSR: (voff, V with global row offsets, E with local ids)."""
    Op, Vp, Ep = u32p(), u32p(), u32p()
    _check(lib.gc_gen_mixed_batch(G, seed0, n_min, n_max, C.byref(Op), C.byref(Vp), C.byref(Ep)),
           what="gen_mixed_batch")
    voff = np.ctypeslib.as_array(Op, shape=(G + 1,)).copy()
    lib.gc_host_free(C.cast(Op, vp))
    N = int(voff[G])
    V = _owned(Vp, N + 1)
    E = _owned(Ep, int(V[N]))
    return voff, V, E


def split_batch(voff: np.ndarray, V: np.ndarray, E: np.ndarray, g: int):
    """Graph g of a segmented CSR as its own (N, V, E) with local ids."""
    a, b = int(voff[g]), int(voff[g + 1])
    Vg = (V[a:b + 1] - V[a]).astype(np.uint32)
    Eg = E[int(V[a]):int(V[b])].copy()
    return b - a, Vg, Eg


def mtx_read(path: str):
    N = C.c_uint32()
    Vp, Ep = u32p(), u32p()
    _check(lib.gc_mtx_read(path.encode(), C.byref(N), C.byref(Vp), C.byref(Ep)), what=f"mtx_read {path}")
    return _take_csr(N.value, Vp, Ep)


def mtx_read_device(ctx: "Context", path: str):
    """gc_mtx_read's CSR, built on the device (gc_mtx_read_device)."""
    N = C.c_uint32()
    Vp, Ep = u32p(), u32p()
    ctx.check(lib.gc_mtx_read_device(ctx.h, str(path).encode(), C.byref(N), C.byref(Vp), C.byref(Ep)),
              f"mtx_read_device {path}")
    return _take_csr(N.value, Vp, Ep)


def mtx_write(path: str, N: int, V: np.ndarray, E: np.ndarray):
    V = np.ascontiguousarray(V, np.uint32)
    E = np.ascontiguousarray(E, np.uint32)
    _check(lib.gc_mtx_write(path.encode(), N, _ptr(V, u32p), _ptr(E, u32p)), what="mtx_write")


# ---- .gnn models -------------------------------------------------------------------------------

def model_read(path: str) -> Tuple[np.ndarray, int]:
    params, md, P = C.c_int(), C.c_int(), f32p()
    _check(lib.gc_model_read(path.encode(), C.byref(params), C.byref(md), C.byref(P)), what=f"model_read {path}")
    arr = np.ctypeslib.as_array(P, shape=(params.value,)).copy()
    lib.gc_host_free(C.cast(P, vp))
    return arr, md.value


def synthetic_model(layers: int, seed: int, md: int = 100) -> Tuple[np.ndarray, int]:
    """Seeded GraphSAGE-16 weights in the .gnn layout: per layer W[32x16] row-major, then b[16].

    Weights ~ N(0, 0.5), biases ~ N(0.1, 0.5), rounded to 10 decimals as .gnn files store them,
    so that writing and re-reading the file gives the same floats."""
    rng = np.random.default_rng(seed)
    P = []
    for _ in range(layers):
        P.append(rng.normal(0.0, 0.5, 512))
        P.append(rng.normal(0.1, 0.5, 16))
    P = np.round(np.concatenate(P), 10)
    return P.astype(np.float32), md


def model_write(path: str, params: np.ndarray, md: int):
    """Writes a .gnn file ("params md" then the floats); the float32 values round-trip exactly."""
    with open(path, "w") as f:
        f.write(f"{len(params)} {md}\n")
        f.write(" ".join(f"{float(x):.9g}" for x in params))
        f.write("\n")


# ---- native device API ---------------------------------------------------------------------------

# Live handles, closed at interpreter exit before module teardown (graphs and models first), so no
# CUDA call runs after the CUDA runtime has shut down.
_live_objects: "weakref.WeakSet" = weakref.WeakSet()
_live_contexts: "weakref.WeakSet" = weakref.WeakSet()


@atexit.register
def _close_all():
    for obj in list(_live_objects):
        try:
            obj.close()
        except Exception:
            pass
    for ctx in list(_live_contexts):
        try:
            ctx.close()
        except Exception:
            pass


class Context:
    def __init__(self, device: int = 0):
        h = vp()
        st = lib.gc_ctx_create(device, C.byref(h))
        if st != 0:
            raise GCError(st, "gc_ctx_create")
        self.h = h
        _live_contexts.add(self)

    def close(self):
        if self.h:
            lib.gc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st, what=""):
        _check(st, self.h, what)

    @property
    def stream(self) -> int:
        return lib.gc_ctx_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(lib.gc_ctx_launches(self.h))

    def sync(self):
        self.check(lib.gc_sync(self.h), "sync")


class Model:
    def __init__(self, ctx: Context, params: np.ndarray, md: int):
        self.ctx = ctx
        params = np.ascontiguousarray(params, np.float32)
        h = vp()
        ctx.check(lib.gc_model_create(ctx.h, len(params), md, _ptr(params, f32p), C.byref(h)), "model")
        self.h = h
        _live_objects.add(self)

    @classmethod
    def load(cls, ctx: Context, path: str) -> "Model":
        params, md = model_read(path)
        return cls(ctx, params, md)

    @property
    def layers(self) -> int:
        return lib.gc_model_layers(self.h)

    def close(self):
        if self.h:
            lib.gc_model_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    @classmethod
    def load_mtx(cls, ctx: Context, path: str) -> "Graph":
        """A Matrix Market file parsed and turned into a CSR on the device (gc_graph_load_mtx)."""
        h = vp()
        ctx.check(lib.gc_graph_load_mtx(ctx.h, str(path).encode(), C.byref(h)), f"load_mtx {path}")
        g = cls.__new__(cls)
        g.ctx, g.h, g.V, g.E = ctx, h, None, None
        g.N = int(lib.gc_graph_num_vertices(h))
        _live_objects.add(g)
        return g

    def __init__(self, ctx: Context, N: int, V: np.ndarray, E: np.ndarray):
        self.ctx = ctx
        self.V = np.ascontiguousarray(V, np.uint32)
        self.E = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
        self.N = int(N)
        h = vp()
        ctx.check(lib.gc_graph_upload(ctx.h, self.N, _ptr(self.V, u32p), _ptr(self.E, u32p), C.byref(h)), "upload")
        self.h = h
        _live_objects.add(self)

    @property
    def M(self) -> int:
        return int(lib.gc_graph_num_edges(self.h))

    @property
    def max_degree(self) -> int:
        return int(lib.gc_graph_max_degree(self.h))

    def priority(self, heuristic, model: Optional[Model] = None):
        h = HEURISTICS[heuristic] if isinstance(heuristic, str) else int(heuristic)
        self.ctx.check(lib.gc_priority(self.ctx.h, self.h, h, model.h if model else None), "priority")

    def set_priority(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float64)
        self.ctx.check(lib.gc_priority_set(self.ctx.h, self.h, _ptr(p, f64p)), "priority_set")

    def color(self, recolor: int = 0, count: bool = True) -> int:
        c = C.c_int(0)
        self.ctx.check(lib.gc_color(self.ctx.h, self.h, recolor, C.byref(c) if count else None), "color")
        return c.value

    def recolor(self, iters: int = 1) -> int:
        c = C.c_int(0)
        self.ctx.check(lib.gc_recolor(self.ctx.h, self.h, iters, C.byref(c)), "recolor")
        return c.value

    def validate(self) -> int:
        c = C.c_int(0)
        self.ctx.check(lib.gc_validate(self.ctx.h, self.h, C.byref(c)), "validate")
        return c.value

    def colors(self) -> np.ndarray:
        out = np.empty(max(self.N, 1), np.int32)
        self.ctx.check(lib.gc_download_colors(self.ctx.h, self.h, _ptr(out, i32p)), "download colors")
        return out[: self.N]

    def set_colors(self, color: np.ndarray):
        color = np.ascontiguousarray(color, np.int32)
        self.ctx.check(lib.gc_upload_colors(self.ctx.h, self.h, _ptr(color, i32p)), "upload colors")

    def priorities(self) -> np.ndarray:
        out = np.empty(max(self.N, 1), np.float64)
        self.ctx.check(lib.gc_download_priority(self.ctx.h, self.h, _ptr(out, f64p)), "download priority")
        return out[: self.N]

    @property
    def device_keys(self) -> int:
        return lib.gc_graph_device_keys(self.h) or 0

    def close(self):
        if self.h:
            lib.gc_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """G independent graphs in one segmented CSR on the device (gc_batch).

    Build it from a segmented CSR (``voff``, global row offsets ``V``, local ids ``E``) or from a list
    of (N, V, E) graphs.  ``color()`` runs priorities + JP (+ Culberson) for all graphs in one CUDA
    graph launch and returns each graph's color count."""

    def __init__(self, ctx: Context, voff: np.ndarray = None, V: np.ndarray = None, E: np.ndarray = None,
                 graphs=None):
        self.ctx = ctx
        h = vp()
        if graphs is not None:
            self._keep = [(np.ascontiguousarray(Vg, np.uint32),
                           np.ascontiguousarray(Eg, np.uint32) if len(Eg) else np.zeros(1, np.uint32))
                          for _, Vg, Eg in graphs]
            G = len(graphs)
            ns = np.array([int(n) for n, _, _ in graphs], np.uint32)
            Vs = (u32p * max(G, 1))(*[_ptr(v, u32p) for v, _ in self._keep])
            Es = (u32p * max(G, 1))(*[_ptr(e, u32p) for _, e in self._keep])
            ctx.check(lib.gc_batch_upload_graphs(ctx.h, G, _ptr(ns, u32p), Vs, Es, C.byref(h)), "batch upload")
            self.voff = np.concatenate([[0], np.cumsum(ns, dtype=np.uint64)]).astype(np.uint32)
            self._keep = None
        else:
            self.voff = np.ascontiguousarray(voff, np.uint32)
            Vc = np.ascontiguousarray(V, np.uint32)
            Ec = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
            G = len(self.voff) - 1
            ctx.check(lib.gc_batch_upload(ctx.h, G, _ptr(self.voff, u32p), _ptr(Vc, u32p), _ptr(Ec, u32p),
                                          C.byref(h)), "batch upload")
        self.h = h
        self.G = G
        _live_objects.add(self)

    @property
    def N(self) -> int:
        return int(lib.gc_batch_num_vertices(self.h))

    @property
    def M(self) -> int:
        return int(lib.gc_batch_num_edges(self.h))

    def color(self, heuristic, model: Optional[Model] = None, recolor: int = 0) -> np.ndarray:
        h = HEURISTICS[heuristic] if isinstance(heuristic, str) else int(heuristic)
        out = np.zeros(max(self.G, 1), np.int32)
        self.ctx.check(lib.gc_batch_color(self.ctx.h, self.h, h, model.h if model else None, recolor,
                                          _ptr(out, i32p)), "batch color")
        return out[: self.G]

    def colors(self) -> np.ndarray:
        out = np.empty(max(self.N, 1), np.int32)
        self.ctx.check(lib.gc_batch_download_colors(self.ctx.h, self.h, _ptr(out, i32p)), "batch colors")
        return out[: self.N]

    def graph_colors(self, g: int, all_colors: Optional[np.ndarray] = None) -> np.ndarray:
        c = self.colors() if all_colors is None else all_colors
        return c[int(self.voff[g]):int(self.voff[g + 1])]

    def priorities(self) -> np.ndarray:
        """Keys of all vertices as doubles (the union graph's gc_download_priority)."""
        out = np.empty(max(self.N, 1), np.float64)
        gh = lib.gc_batch_graph(self.h)
        self.ctx.check(lib.gc_download_priority(self.ctx.h, gh, _ptr(out, f64p)), "batch priorities")
        return out[: self.N]

    def autotune(self, heuristic, model: Optional[Model] = None, recolor: int = 0, effort: int = 1):
        h = HEURISTICS[heuristic] if isinstance(heuristic, str) else int(heuristic)
        t = Tuning()
        ms = C.c_double(0.0)
        self.ctx.check(lib.gc_batch_autotune(self.ctx.h, self.h, h, model.h if model else None, recolor, effort,
                                             C.byref(t), C.byref(ms)), "autotune")
        return t, ms.value

    @property
    def tuning(self) -> Tuning:
        t = Tuning()
        _check(lib.gc_batch_get_tuning(self.h, C.byref(t)), what="get tuning")
        return t

    @tuning.setter
    def tuning(self, t: Tuning):
        self.ctx.check(lib.gc_batch_set_tuning(self.ctx.h, self.h, C.byref(t)), "set tuning")

    def close(self):
        if self.h:
            lib.gc_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """A coloring server on one GPU (gc_server): continuous batching over device-resident pools,
    admission by HBM budget, per-job latency.  Each job's colors equal its graph colored alone.

    ``submit`` keeps references to the job's arrays until ``wait`` returns, as the C API requires
    the caller's buffers to stay valid until the job is done."""

    def __init__(self, device: int = 0, lanes: int = 4, hbm_budget: int = 0, slot_graphs: int = 4096,
                 slot_vertices: int = 1 << 22, slot_edges: int = 1 << 26, batch_max_job_vertices: int = 1 << 17,
                 models=()):
        cfg = ServeConfig()
        lib.gc_serve_config_default(C.byref(cfg))
        cfg.device, cfg.lanes, cfg.hbm_budget = device, lanes, hbm_budget
        cfg.slot_graphs, cfg.slot_vertices, cfg.slot_edges = slot_graphs, slot_vertices, slot_edges
        cfg.batch_max_job_vertices = batch_max_job_vertices
        h = vp()
        st = lib.gc_serve_create(C.byref(cfg), C.byref(h))
        if st != 0:
            raise GCError(st, "gc_serve_create")
        self.h = h
        self._held = {}
        self._reg_n = {}
        _live_objects.add(self)
        for params, md in models:
            self.add_model(params, md)

    def _check(self, st, what):
        if st != 0:
            detail = lib.gc_serve_last_error(self.h) if self.h else b""
            raise GCError(st, f"{what}: {detail.decode()}" if detail else what)

    def add_model(self, params: np.ndarray, md: int):
        p = np.ascontiguousarray(params, np.float32)
        self._check(lib.gc_serve_add_model(self.h, len(p), md, _ptr(p, f32p)), "add model")

    @staticmethod
    def _job_arrays(N, V, E):
        Vc = np.ascontiguousarray(V, np.uint32)
        Ec = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
        return Vc, Ec

    def submit(self, N: int, V: np.ndarray, E: np.ndarray, heuristic="FF", layers: int = 0, recolor: int = 0,
               want_colors: bool = True) -> int:
        h = HEURISTICS[heuristic] if isinstance(heuristic, str) else int(heuristic)
        Vc, Ec = self._job_arrays(N, V, E)
        out = np.zeros(max(int(N), 1), np.int32) if want_colors else None
        jid = C.c_uint64(0)
        self._check(lib.gc_serve_submit(self.h, int(N), _ptr(Vc, u32p), _ptr(Ec, u32p), h, layers, recolor,
                                        _ptr(out, i32p) if out is not None else None, C.byref(jid)), "submit")
        self._held[jid.value] = (Vc, Ec, out, int(N))
        return jid.value

    def register(self, N: int, V: np.ndarray, E: np.ndarray) -> int:
        """Uploads a CSR once; returns its id for submit_registered / replay_registered."""
        Vc, Ec = self._job_arrays(N, V, E)
        gid = C.c_uint64(0)
        self._check(lib.gc_serve_register(self.h, int(N), _ptr(Vc, u32p), _ptr(Ec, u32p), C.byref(gid)), "register")
        self._reg_n[gid.value] = int(N)
        return gid.value

    def unregister(self, graph: int):
        self._check(lib.gc_serve_unregister(self.h, graph), "unregister")
        self._reg_n.pop(graph, None)

    def submit_registered(self, graph: int, heuristic="FF", layers: int = 0, recolor: int = 0,
                          want_colors: bool = True) -> int:
        h = HEURISTICS[heuristic] if isinstance(heuristic, str) else int(heuristic)
        N = self._reg_n[graph]
        out = np.zeros(max(N, 1), np.int32) if want_colors else None
        jid = C.c_uint64(0)
        self._check(lib.gc_serve_submit_registered(self.h, graph, h, layers, recolor,
                                                   _ptr(out, i32p) if out is not None else None, C.byref(jid)),
                    "submit registered")
        self._held[jid.value] = (None, None, out, N)
        return jid.value

    def replay_registered(self, arrive_s, graphs, heuristics, layers=None, recolor=None, want_colors: bool = False):
        """Open-loop load on registered graphs: job i runs on graphs[i] (an id) at arrive_s[i] seconds."""
        J = len(graphs)
        arr = np.ascontiguousarray(arrive_s, np.float64)
        ids = (C.c_uint64 * max(J, 1))(*[int(g) for g in graphs])
        hs = np.array([HEURISTICS[x] if isinstance(x, str) else int(x) for x in heuristics], np.int32)
        ls = np.array(layers if layers is not None else [0] * J, np.int32)
        rs = np.array(recolor if recolor is not None else [0] * J, np.int32)
        outs = [np.zeros(max(self._reg_n[int(g)], 1), np.int32) for g in graphs] if want_colors else None
        op = (i32p * max(J, 1))(*[_ptr(o, i32p) for o in outs]) if want_colors else None
        infos = (JobInfo * max(J, 1))()
        i32 = C.POINTER(C.c_int)
        st = lib.gc_serve_replay_registered(self.h, J, _ptr(arr, f64p), ids, hs.ctypes.data_as(i32),
                                            ls.ctypes.data_as(i32), rs.ctypes.data_as(i32), op, infos)
        self._check(st, "replay registered")
        cols = [o[: self._reg_n[int(g)]] for o, g in zip(outs, graphs)] if want_colors else None
        return cols, [infos[i].as_dict() for i in range(J)]

    def done(self, job: int) -> bool:
        d = C.c_int(0)
        self._check(lib.gc_serve_test(self.h, job, C.byref(d)), "test")
        return bool(d.value)

    def wait(self, job: int):
        """(colors or None, JobInfo); raises GCError when the job failed."""
        info = JobInfo()
        st = lib.gc_serve_wait(self.h, job, C.byref(info))
        Vc, Ec, out, N = self._held.pop(job, (None, None, None, 0))
        self._check(st, f"job {job}")
        return (out[:N] if out is not None else None), info

    def drain(self):
        self._check(lib.gc_serve_drain(self.h), "drain")

    def replay(self, arrive_s, graphs, heuristics, layers=None, recolor=None, want_colors: bool = False):
        """Open-loop load: graphs[i] = (N, V, E) arrives at arrive_s[i] seconds.  Returns
        (list of colors or None, list of JobInfo dicts)."""
        J = len(graphs)
        keep = [self._job_arrays(*g) for g in graphs]
        arr = np.ascontiguousarray(arrive_s, np.float64)
        ns = np.array([int(g[0]) for g in graphs], np.uint32)
        Vs = (u32p * max(J, 1))(*[_ptr(v, u32p) for v, _ in keep])
        Es = (u32p * max(J, 1))(*[_ptr(e, u32p) for _, e in keep])
        hs = np.array([HEURISTICS[x] if isinstance(x, str) else int(x) for x in heuristics], np.int32)
        ls = np.array(layers if layers is not None else [0] * J, np.int32)
        rs = np.array(recolor if recolor is not None else [0] * J, np.int32)
        outs = [np.zeros(max(int(g[0]), 1), np.int32) for g in graphs] if want_colors else None
        op = (i32p * max(J, 1))(*[_ptr(o, i32p) for o in outs]) if want_colors else None
        infos = (JobInfo * max(J, 1))()
        i32 = C.POINTER(C.c_int)
        st = lib.gc_serve_replay(self.h, J, _ptr(arr, f64p), _ptr(ns, u32p), Vs, Es, hs.ctypes.data_as(i32),
                                 ls.ctypes.data_as(i32), rs.ctypes.data_as(i32), op, infos)
        self._check(st, "replay")
        cols = [o[: int(g[0])] for o, g in zip(outs, graphs)] if want_colors else None
        return cols, [infos[i].as_dict() for i in range(J)]

    def stats(self) -> dict:
        st = ServeStats()
        self._check(lib.gc_serve_read_stats(self.h, C.byref(st)), "stats")
        return st.as_dict()

    def reset_stats(self):
        lib.gc_serve_reset_stats(self.h)

    def close(self):
        if self.h:
            lib.gc_serve_destroy(self.h)
            self.h = None
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_config_default() -> ServeConfig:
    c = ServeConfig()
    lib.gc_serve_config_default(C.byref(c))
    return c


def default_tuning() -> Tuning:
    t = Tuning()
    lib.gc_tuning_default(C.byref(t))
    return t


def batch_device_bytes(G: int, N: int, M: int, heuristic) -> int:
    h = HEURISTICS[heuristic] if isinstance(heuristic, str) else int(heuristic)
    return int(lib.gc_batch_device_bytes(G, N, M, h))


# ---- the reference-named drop-in functions ------------------------------------------------------

class _Legacy:
    """numpy front-end of the reference's own entry points, as exported by libgnncolor.so."""

    def __init__(self):
        for name in ("first_fit_ordering", "first_fit_ordering_par", "largest_degree_first_ordering",
                     "largest_log_degree_first_ordering", "smallest_degree_last_ordering",
                     "smallest_log_degree_last_ordering"):
            _sig(name, None, C.c_uint32, u32p, u32p, f64p)
        _sig("gnn_ordering", None, C.c_uint32, u32p, u32p, f64p, C.c_int)
        for name in ("jones_plassmann_coloring", "greedy_coloring"):
            _sig(name, i32p, C.c_uint32, u32p, u32p, f64p)
        for name in ("first_fit_coloring", "first_fit_coloring_par", "largest_degree_first_coloring",
                     "largest_degree_first_coloring_par", "largest_log_degree_first_coloring",
                     "largest_log_degree_first_coloring_par", "smallest_degree_last_coloring",
                     "smallest_degree_last_coloring_par", "smallest_log_degree_last_coloring",
                     "smallest_log_degree_last_coloring_par"):
            _sig(name, i32p, C.c_uint32, u32p, u32p)
        for name in ("validate_coloring", "validate_coloring_par"):
            _sig(name, C.c_int, C.c_uint32, u32p, u32p, i32p)
        for name in ("jones_plassmann_setup", "greedy_setup", "gnn_setup", "first_fit_setup"):
            _sig(name, vp, C.c_uint32, C.c_uint32)
        for name in ("jones_plassmann_cleanup", "greedy_cleanup", "gnn_cleanup", "first_fit_cleanup"):
            _sig(name, None, vp)
        for name in ("jones_plassmann_internal", "greedy_internal"):
            _sig(name, None, C.c_uint32, u32p, u32p, vp, f64p, i32p)
        for name in ("gnn_internal_par", "gnn_internal", "first_fit_internal_par"):
            _sig(name, None, C.c_uint32, u32p, u32p, vp, vp, f64p, i32p)
        for name in ("cgnn_graph_sage_16", "cgnn_graph_sage_16_par"):
            _sig(name, None, C.c_int, f32p, C.c_uint32, u32p, u32p, C.c_int, f32p, f32p, f64p)
        self.libc = C.CDLL(None)
        self.libc.free.argtypes = [vp]

    @staticmethod
    def _csr(V, E):
        V = np.ascontiguousarray(V, np.uint32)
        E = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
        return V, E

    def ordering(self, name: str, N, V, E, layers: int = 0) -> np.ndarray:
        V, E = self._csr(V, E)
        p = np.zeros(N + 8, np.float64)
        if name == "gnn_ordering":
            lib.gnn_ordering(N, _ptr(V, u32p), _ptr(E, u32p), _ptr(p, f64p), layers)
        else:
            getattr(lib, name)(N, _ptr(V, u32p), _ptr(E, u32p), _ptr(p, f64p))
        return p[:N]

    def _take(self, ptr, N) -> np.ndarray:
        out = np.ctypeslib.as_array(ptr, shape=(max(N, 1),))[:N].copy()
        self.libc.free(C.cast(ptr, vp))
        return out

    def coloring(self, name: str, N, V, E, p: Optional[np.ndarray] = None) -> np.ndarray:
        V, E = self._csr(V, E)
        if p is None:
            ptr = getattr(lib, name)(N, _ptr(V, u32p), _ptr(E, u32p))
        else:
            p = np.ascontiguousarray(p, np.float64)
            ptr = getattr(lib, name)(N, _ptr(V, u32p), _ptr(E, u32p), _ptr(p, f64p))
        return self._take(ptr, N)

    def validate(self, N, V, E, color) -> int:
        V, E = self._csr(V, E)
        color = np.ascontiguousarray(color, np.int32)
        return lib.validate_coloring_par(N, _ptr(V, u32p), _ptr(E, u32p), _ptr(color, i32p))

    def graph_sage(self, params: np.ndarray, md: int, N, V, E) -> np.ndarray:
        V, E = self._csr(V, E)
        params = np.ascontiguousarray(params, np.float32)
        p = np.zeros(N + 8, np.float64)
        lib.cgnn_graph_sage_16_par(len(params), _ptr(params, f32p), N, _ptr(V, u32p), _ptr(E, u32p), md, None,
                                   None, _ptr(p, f64p))
        return p[:N]


legacy = _Legacy()
