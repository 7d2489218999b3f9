"""ctypes loader of the reference's own C code (oracle/_ref/libref.so, built by oracle/Makefile
from the reference's unchanged sources).  Used to pin the oracle, to generate golden vectors and
as the timed CPU baseline.  Test/bench infrastructure only.

The reference's fast_gnn.c uses aligned AVX loads and streaming stores on x, y and p, so every
buffer handed to it here is 64-byte aligned and padded by 8 rows, as fast_gnn.h:4-11 asks."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libref.so")
MODELS = os.path.join(HERE, "_ref", "models")


def available() -> bool:
    return os.path.exists(PATH)


u32p, i32p, f32p, f64p = (C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_float),
                          C.POINTER(C.c_double))
vp = C.c_void_p
_lib = None
_gomp = None


def lib():
    global _lib, _gomp
    if _lib is None:
        if not available():
            raise ImportError(f"{PATH} missing: run `make -C {HERE}` where the reference sources exist")
        _lib = C.CDLL(PATH)
        _gomp = C.CDLL("libgomp.so.1")
        for name in ("first_fit_ordering", "first_fit_ordering_par", "largest_degree_first_ordering",
                     "largest_log_degree_first_ordering", "largest_log_degree_first_ordering_par",
                     "smallest_degree_last_ordering", "smallest_log_degree_last_ordering"):
            getattr(_lib, name).argtypes = [C.c_uint32, u32p, u32p, vp]
        for name in ("cgnn_graph_sage_16", "cgnn_graph_sage_16_par"):
            getattr(_lib, name).argtypes = [C.c_int, vp, C.c_uint32, u32p, u32p, C.c_int, vp, vp, vp]
        for name in ("jones_plassmann_coloring", "greedy_coloring"):
            getattr(_lib, name).argtypes = [C.c_uint32, u32p, u32p, vp]
            getattr(_lib, name).restype = i32p
        for name in ("jones_plassmann_setup", "greedy_setup", "smallest_degree_last_setup"):
            getattr(_lib, name).argtypes = [C.c_uint32, C.c_uint32]
            getattr(_lib, name).restype = vp
        for name in ("jones_plassmann_cleanup", "greedy_cleanup", "smallest_degree_last_cleanup"):
            getattr(_lib, name).argtypes = [vp]
        for name in ("jones_plassmann_internal", "greedy_internal"):
            getattr(_lib, name).argtypes = [C.c_uint32, u32p, u32p, vp, vp, i32p]
        for name in ("smallest_degree_last_internal_par", "smallest_log_degree_last_internal_par"):
            getattr(_lib, name).argtypes = [C.c_uint32, u32p, u32p, vp, vp, vp, i32p]
        _lib.validate_coloring_par.argtypes = [C.c_uint32, u32p, u32p, i32p]
        _lib.validate_coloring_par.restype = C.c_int
        _gomp.omp_set_num_threads.argtypes = [C.c_int]
        _gomp.omp_get_max_threads.restype = C.c_int
    return _lib


def set_threads(n: int):
    lib()
    _gomp.omp_set_num_threads(int(n))


def max_threads() -> int:
    lib()
    return int(_gomp.omp_get_max_threads())


def aligned(n: int, dtype) -> np.ndarray:
    """Zeroed array of n elements whose data starts on a 64-byte boundary."""
    itemsize = np.dtype(dtype).itemsize
    raw = np.zeros(n * itemsize + 64, np.uint8)
    off = (-raw.ctypes.data) % 64
    return raw[off:off + n * itemsize].view(dtype)


def _csr(V, E):
    V = np.ascontiguousarray(V, np.uint32)
    E = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
    return V, E, V.ctypes.data_as(u32p), E.ctypes.data_as(u32p)


def ordering(name: str, N: int, V, E) -> np.ndarray:
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    p = aligned(N + 8, np.float64)
    fn = {"FF": "first_fit_ordering_par", "LF": "largest_degree_first_ordering",
          "LLF": "largest_log_degree_first_ordering", "SL": "smallest_degree_last_ordering",
          "SLL": "smallest_log_degree_last_ordering"}[name]
    getattr(L, fn)(N, Vp, Ep, p.ctypes.data)
    return p[:N].copy()


def peel_par(name: str, N: int, V, E) -> tuple[np.ndarray, np.ndarray]:
    """The parallel SL/SLL variants (smallest_degree_last.c:155-246, :359-443): p and colors."""
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    p = aligned(N + 8, np.float64)
    color = np.zeros(max(N, 1), np.int32)
    sl = L.smallest_degree_last_setup(N, int(V[N]))
    jp = L.jones_plassmann_setup(N, int(V[N]))
    fn = L.smallest_degree_last_internal_par if name == "SL" else L.smallest_log_degree_last_internal_par
    fn(N, Vp, Ep, sl, jp, p.ctypes.data, color.ctypes.data_as(i32p))
    L.smallest_degree_last_cleanup(sl)
    L.jones_plassmann_cleanup(jp)
    return p[:N].copy(), color[:N].copy()


def graph_sage(params: np.ndarray, md: int, N: int, V, E) -> np.ndarray:
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    P = aligned(len(params), np.float32)
    P[:] = params
    x = aligned((N + 8) * 16, np.float32)
    y = aligned((N + 8) * 16, np.float32)
    p = aligned(N + 8, np.float64)
    L.cgnn_graph_sage_16_par(len(params), P.ctypes.data, N, Vp, Ep, md, x.ctypes.data, y.ctypes.data, p.ctypes.data)
    return p[:N].copy()


def jp_color(N: int, V, E, p) -> np.ndarray:
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    pp = aligned(N + 8, np.float64)
    pp[:N] = p
    c = L.jones_plassmann_coloring(N, Vp, Ep, pp.ctypes.data)
    out = np.ctypeslib.as_array(c, shape=(max(N, 1),))[:N].copy()
    C.CDLL(None).free(C.cast(c, vp))
    return out


def greedy_color_defined(N: int, V, E, p) -> np.ndarray:
    """The reference's greedy_internal (coloring.c:60-125) with its uninitialized reads made
    deterministic.  Its mex loop reads marks[c] for c up to max_degree + 1, but only entries
    0..max_degree are initialized (coloring.c:89-90), and marks holds only N entries.  Here the
    state is set up for N + 2 vertices and marks is filled with 0xFFFFFFFF (never a vertex id)
    before the call, so those reads see "not marked", which is what the algorithm means."""
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    if N == 0:
        return np.zeros(0, np.int32)
    pp = aligned(N + 8, np.float64)
    pp[:N] = p
    color = np.zeros(N, np.int32)
    gd = L.greedy_setup(N + 2, max(int(V[N]), 1))
    # struct gd_data { uint32_t *next, *prev, *count, *pred, *E_split, *marks; } (coloring.c:18-24)
    marks = C.cast(gd, C.POINTER(C.c_void_p))[5]
    C.memset(marks, 0xFF, 4 * (N + 2))
    L.greedy_internal(N, Vp, Ep, gd, pp.ctypes.data, color.ctypes.data_as(i32p))
    L.greedy_cleanup(gd)
    return color


def greedy_color(N: int, V, E, p) -> np.ndarray:
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    pp = aligned(N + 8, np.float64)
    pp[:N] = p
    c = L.greedy_coloring(N, Vp, Ep, pp.ctypes.data)
    out = np.ctypeslib.as_array(c, shape=(max(N, 1),))[:N].copy()
    C.CDLL(None).free(C.cast(c, vp))
    return out


def has_models() -> bool:
    return all(os.path.exists(os.path.join(MODELS, f"m{L}.gnn")) for L in (2, 3, 4))


class GnnJob:
    """The reference's GNN heuristic as its runner drives it: gnn_setup reads models/m{L}.gnn
    relative to the working directory (src/gnn.c:24-25), so the call runs from _ref/, where
    oracle/Makefile copies the reference's model files; gnn_internal_par (gnn.c:78-83) then gives
    p and the JP colors, and each Culberson round sets p := color and re-runs
    jones_plassmann_internal (src/runner.c:139-152)."""

    def __init__(self, N: int, V, E, layers: int):
        L = lib()
        L.gnn_setup.argtypes = [C.c_uint32, C.c_uint32]
        L.gnn_setup.restype = vp
        L.gnn_internal_par.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp]
        L.gnn_cleanup.argtypes = [vp]
        self.N = N
        self.V = np.ascontiguousarray(V, np.uint32)
        self.E = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
        M = int(self.V[N])
        C.c_int.in_dll(L, "layers").value = int(layers)
        cwd = os.getcwd()
        os.chdir(os.path.join(HERE, "_ref"))
        try:
            self.ad = L.gnn_setup(N, M)
        finally:
            os.chdir(cwd)
        self.jp = L.jones_plassmann_setup(N, M)
        self.p = aligned(N + 8, np.float64)
        self.color = np.zeros(max(N, 1), np.int32)

    def run(self):
        """One f_par call: GNN priorities + JP.  Returns the colors (a view, overwritten by the next
        call)."""
        lib().gnn_internal_par(self.N, self.V.ctypes.data, self.E.ctypes.data, self.ad, self.jp,
                               self.p.ctypes.data, self.color.ctypes.data)
        return self.color

    def culberson(self):
        """One recoloring round: p := color, then the reference's JP."""
        self.p[:self.N] = self.color[:self.N]
        lib().jones_plassmann_internal(self.N, self.V.ctypes.data_as(u32p), self.E.ctypes.data_as(u32p), self.jp,
                                       self.p.ctypes.data, self.color.ctypes.data_as(i32p))
        return self.color

    def close(self):
        if self.ad:
            lib().gnn_cleanup(self.ad)
            lib().jones_plassmann_cleanup(self.jp)
            self.ad = None


def csr_from_samples(N: int, I, J):
    """The reference's own graph construction from 0-based edge samples: mtx_to_graph_par (both
    directions of every entry, src/fast_io.c:171-202), graph_sort_edges_par and graph_make_simple
    (fast_io.c:450-477).  Returns (V, E) as numpy copies."""
    L = lib()
    fn = L.mtx_to_graph_par
    fn.argtypes = [C.c_uint32, u32p, u32p, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p)]
    L.graph_sort_edges_par.argtypes = [C.c_uint32, u32p, u32p]
    L.graph_make_simple.argtypes = [C.c_uint32, u32p, C.POINTER(u32p)]
    I1 = np.ascontiguousarray(I, np.uint32) + np.uint32(1)
    J1 = np.ascontiguousarray(J, np.uint32) + np.uint32(1)
    Vp, Ep = u32p(), u32p()
    fn(len(I1), I1.ctypes.data_as(u32p), J1.ctypes.data_as(u32p), N, C.byref(Vp), C.byref(Ep))
    del I1, J1
    L.graph_sort_edges_par(N, Vp, Ep)
    L.graph_make_simple(N, Vp, C.byref(Ep))
    V = np.ctypeslib.as_array(Vp, shape=(N + 1,)).copy()
    M = int(V[N])
    E = np.ctypeslib.as_array(Ep, shape=(max(M, 1),))[:M].copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [vp]
    libc.free(C.cast(Vp, vp))
    libc.free(C.cast(Ep, vp))
    return V, E


def validate(N: int, V, E, color) -> int:
    L = lib()
    V, E, Vp, Ep = _csr(V, E)
    color = np.ascontiguousarray(color, np.int32)
    return int(L.validate_coloring_par(N, Vp, Ep, color.ctypes.data_as(i32p)))
