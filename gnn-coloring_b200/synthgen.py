"""Seeded R-MAT edge samples in numpy, without loading libgnncolor.so.

The library's generator (csrc/host_graph.cpp, gc_gen_rmat) draws sample k from its own
SplitMix64 stream keyed by (seed, k): one uniform double per bit of the vertex ids, lowest bit
first, with the quadrant picked by comparing that double against a, a + b and a + b + c.  This
module draws the identical samples with vectorised uint64 arithmetic, so that a process which must
not map the library (the timed run of the reference's own CPU code) still colors the same graph.

Only the samples are produced here.  Turning them into a CSR is left to the caller: the reference
arm hands them, 1-based, to the reference's own mtx_to_graph_par + graph_sort_edges_par +
graph_make_simple (src/fast_io.c:171-202, 450-477), which apply the same rules as the library's
gc_csr_build.  tests/test_host.py checks both CSRs are equal.
"""
from __future__ import annotations

import math
import multiprocessing as mp
import os

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_MASK = (1 << 64) - 1


def _mix_py(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
    return z ^ (z >> 31)


def _stream_key(seed: int) -> int:
    """First output of the seed's SplitMix64 state; host_graph.cpp stream_state XORs it with the
    scaled sample index."""
    s = (seed * 0xD1B54A32D192ED03 + 0x2545F4914F6CDD1D) & _MASK
    s = (s + 0x9E3779B97F4A7C15) & _MASK
    return _mix_py(s)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def _rmat_chunk(args):
    k0, k1, scale, seed, a, b, c = args
    key = np.uint64(_stream_key(seed))
    with np.errstate(over="ignore"):
        k = np.arange(k0, k1, dtype=np.uint64)
        # state after stream_state(seed, k): (key ^ k * golden) advanced once
        s = (key ^ (k * GOLDEN)) + GOLDEN
        del k
        ab, abc = a + b, a + b + c
        u = np.zeros(k1 - k0, np.uint64)
        v = np.zeros(k1 - k0, np.uint64)
        for bit in range(scale):
            s += GOLDEN
            r = (_mix(s) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
            ub = r >= ab
            vb = ((r >= a) & (r < ab)) | (r >= abc)
            u |= ub.astype(np.uint64) << np.uint64(bit)
            v |= vb.astype(np.uint64) << np.uint64(bit)
    return u, v


def _rmat_kept(args):
    n = args[0]
    u, v = _rmat_chunk(args[1:])
    keep = (u < n) & (v < n)
    return u[keep].astype(np.uint32), v[keep].astype(np.uint32)


def rmat_samples(n: int, ef: float, seed: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                 workers: int = 0):
    """The kept samples (I, J) of gc_gen_rmat(n, ef, a, b, c, seed) as uint32 arrays, in sample
    order (self-loops and repeats included: the CSR build drops them).  `workers` > 1 spreads the
    sample range over spawned processes (numpy only)."""
    scale = 0
    while scale < 32 and (1 << scale) < n:
        scale += 1
    samples = int(math.floor(ef * n + 0.5))  # llround (halves away from zero) for ef * n >= 0
    if workers <= 0:
        workers = min(16, os.cpu_count() or 1)
    chunk = 1 << 21
    tasks = [(n, k0, min(samples, k0 + chunk), scale, seed, a, b, c) for k0 in range(0, samples, chunk)]
    if workers > 1 and len(tasks) > 1:
        with mp.get_context("spawn").Pool(min(workers, len(tasks))) as pool:
            parts = pool.map(_rmat_kept, tasks)
    else:
        parts = [_rmat_kept(t) for t in tasks]
    if not parts:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])
