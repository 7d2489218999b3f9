"""ctypes loader of liboracle.so, the scalar C restatement of the reference (oracle.c).

Test infrastructure: the checker, never the product path."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "liboracle.so")
if not os.path.exists(PATH):
    raise ImportError(f"{PATH} missing: run `make -C {HERE}`")
_lib = C.CDLL(PATH)
u32p, i32p, f32p, f64p = (C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_float),
                          C.POINTER(C.c_double))
for name in ("oracle_ff_ordering", "oracle_lf_ordering", "oracle_llf_ordering"):
    getattr(_lib, name).argtypes = [C.c_uint32, u32p, f64p]
for name in ("oracle_sl_ordering", "oracle_sll_ordering"):
    getattr(_lib, name).argtypes = [C.c_uint32, u32p, u32p, f64p]
for name in ("oracle_gnn_ordering", "oracle_gnn_ordering_f64"):
    getattr(_lib, name).argtypes = [C.c_int, f32p, C.c_int, C.c_uint32, u32p, u32p, f64p]
_lib.oracle_greedy_color.argtypes = [C.c_uint32, u32p, u32p, f64p, i32p]
_lib.oracle_greedy_color.restype = C.c_uint32
_lib.oracle_culberson.argtypes = [C.c_uint32, u32p, u32p, f64p, i32p, C.c_int]
_lib.oracle_validate.argtypes = [C.c_uint32, u32p, u32p, i32p]
_lib.oracle_validate.restype = C.c_int


def _csr(V, E):
    V = np.ascontiguousarray(V, np.uint32)
    E = np.ascontiguousarray(E, np.uint32) if len(E) else np.zeros(1, np.uint32)
    return V, E, V.ctypes.data_as(u32p), E.ctypes.data_as(u32p)


def ordering(name: str, N: int, V, E, params=None, md: int = 100) -> np.ndarray:
    """Priorities of heuristic `name` (FF, LF, LLF, SL, SLL, GNN, GNN64) as the reference's doubles."""
    V, E, Vp, Ep = _csr(V, E)
    p = np.zeros(max(N, 1), np.float64)
    pp = p.ctypes.data_as(f64p)
    if name == "FF":
        _lib.oracle_ff_ordering(N, Vp, pp)
    elif name == "LF":
        _lib.oracle_lf_ordering(N, Vp, pp)
    elif name == "LLF":
        _lib.oracle_llf_ordering(N, Vp, pp)
    elif name == "SL":
        _lib.oracle_sl_ordering(N, Vp, Ep, pp)
    elif name == "SLL":
        _lib.oracle_sll_ordering(N, Vp, Ep, pp)
    elif name in ("GNN", "GNN64"):
        P = np.ascontiguousarray(params, np.float32)
        f = _lib.oracle_gnn_ordering if name == "GNN" else _lib.oracle_gnn_ordering_f64
        f(len(P), P.ctypes.data_as(f32p), md, N, Vp, Ep, pp)
    else:
        raise ValueError(name)
    return p[:N]


def greedy_color(N: int, V, E, p) -> tuple[np.ndarray, int]:
    """Colors (1-based) of the priority-order greedy, and the number of peeling rounds."""
    V, E, Vp, Ep = _csr(V, E)
    p = np.ascontiguousarray(p, np.float64)
    if N == 0:
        return np.zeros(0, np.int32), 0
    color = np.zeros(N, np.int32)
    rounds = _lib.oracle_greedy_color(N, Vp, Ep, p.ctypes.data_as(f64p), color.ctypes.data_as(i32p))
    return color, int(rounds)


def culberson(N: int, V, E, color, iters: int) -> np.ndarray:
    V, E, Vp, Ep = _csr(V, E)
    color = np.array(color, np.int32, copy=True)
    if N == 0 or iters == 0:
        return color
    p = np.zeros(N, np.float64)
    _lib.oracle_culberson(N, Vp, Ep, p.ctypes.data_as(f64p), color.ctypes.data_as(i32p), iters)
    return color


def validate(N: int, V, E, color) -> int:
    V, E, Vp, Ep = _csr(V, E)
    color = np.ascontiguousarray(color, np.int32) if N else np.zeros(1, np.int32)
    return int(_lib.oracle_validate(N, Vp, Ep, color.ctypes.data_as(i32p)))
