"""Generates the golden vectors in this directory by running the reference's own C code.

The reference (KennethLangedal/GNN-COLORING) ships no tests or fixtures besides its model files,
so its outputs on seeded synthetic graphs are the golden vectors.  This script needs
oracle/_ref/libref.so, which oracle/Makefile compiles from the reference's unchanged sources
(only where the reference tree is present); the committed .npz files then travel without it.

  golden_synth.npz      priorities p and JP colors of all 8 heuristics, with seeded synthetic
                        GraphSAGE weights (GNN2/3/4), plus colors after 3 Culberson recolorings;
                        for several small graphs and hand-built edge cases.  Graphs are stored too.
  golden_refmodels.npz  GNN2/3/4 priorities and colors with the reference's own model files
                        (models/m{2,3,4}.gnn); the weights themselves are not stored.
  golden_incidence.npz  the reference's ID, SDA and SD priorities (src/incidence_degree.c) and JP
                        colors on the same graphs
  golden_formats.npz    texts written by the reference's mtx/adj/gr/metis writers and what its
                        adj/gr/metis readers return for them
  golden_mtx.npz        the reference's CSR (mtx_parse_par + graph_sort_edges_par +
                        graph_make_simple) of small Matrix Market texts with duplicates,
                        self-loops, one-sided entries, comments and value columns.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "gnn-coloring_b200"))

import gnn_coloring as gcn  # noqa: E402  (host generators only; no GPU needed)
from oracle import reference as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def edge_case_graphs():
    """Small graphs that exercise the reference's corner cases."""
    g = {}

    def from_pairs(n, pairs):
        if pairs:
            I, J = np.array(pairs, np.uint32).T
        else:
            I = J = np.zeros(0, np.uint32)
        return gcn.csr_from_pairs(n, I, J)

    g["path7"] = from_pairs(7, [(i, i + 1) for i in range(6)])
    g["star9"] = from_pairs(9, [(0, i) for i in range(1, 9)])
    g["clique6"] = from_pairs(6, [(i, j) for i in range(6) for j in range(i + 1, 6)])
    g["isolated5"] = from_pairs(5, [])
    g["tiny3"] = from_pairs(3, [(0, 2)])
    g["single1"] = from_pairs(1, [])
    # equal degrees everywhere: every integer heuristic is decided by the id tie rule
    g["cycle12"] = from_pairs(12, [(i, (i + 1) % 12) for i in range(12)])
    # two cliques joined by a path, plus isolated vertices at both ends of the id range
    pairs = [(i, j) for i in range(1, 6) for j in range(i + 1, 6)]
    pairs += [(i, j) for i in range(10, 16) for j in range(i + 1, 16)]
    pairs += [(5, 6), (6, 7), (7, 8), (8, 9), (9, 10)]
    g["bridged"] = from_pairs(18, pairs)
    return g


def synth_graphs():
    g = {}
    g["er1500"] = gcn.gen_er(1500, 6000, 7)
    g["rmat11"] = gcn.gen_rmat(2048, 8, 3)
    g["rgg2k"] = gcn.gen_rgg2d(2000, float(np.sqrt(12 / (np.pi * 2000))), 5)
    g["stencil6"] = gcn.gen_stencil27(6, 5, 4)
    return g


SYNTH_MODEL_SEEDS = {2: 1002, 3: 1003, 4: 1004}


def jp_color(N, V, E, p):
    """The reference's coloring of p.  Its mex loop reads marks[max_degree + 1], an entry it never
    initialized (coloring.c:89-90 and :279-280 set only max_degree + 1 entries; with N entries in
    all, a clique even reads past the block), so the raw output depends on leftover memory.  The
    golden colors come from the reference's greedy_internal run with that entry made
    deterministic (oracle/reference.py: greedy_color_defined).  Where the reference's JP does not
    hit the uninitialized entry its colors are checked to agree."""
    c = R.greedy_color_defined(N, V, E, p)
    if N and int(V[N]) and c.max() <= int(np.diff(V.astype(np.int64)).max()):
        assert np.array_equal(c, R.jp_color(N, V, E, p))
    return c


def run_heuristics(store, name, N, V, E, models):
    for h in ("FF", "LF", "LLF", "SL", "SLL"):
        p = R.ordering(h, N, V, E)
        c = jp_color(N, V, E, p)
        if h in ("SL", "SLL"):
            pp, cp = R.peel_par(h, N, V, E)
            assert np.array_equal(pp, p), (name, h, "parallel peel differs")
        store[f"{name}/{h}/p"] = p
        store[f"{name}/{h}/color"] = c
        store[f"{name}/{h}/culb3"] = culberson(N, V, E, c, 3)
    for L, (params, md) in models.items():
        p = R.graph_sage(params, md, N, V, E)
        c = jp_color(N, V, E, p)
        store[f"{name}/GNN{L}/p"] = p
        store[f"{name}/GNN{L}/color"] = c
        store[f"{name}/GNN{L}/culb3"] = culberson(N, V, E, c, 3)


def culberson(N, V, E, color, iters):
    c = color.copy()
    for _ in range(iters):
        c = jp_color(N, V, E, c.astype(np.float64))
    return c


MTX_CASES = {
    "dups_loops": "%%MatrixMarket matrix coordinate pattern symmetric\n% comment\n6 6 9\n"
                  "2 1\n3 1\n3 3\n4 2\n2 1\n6 5\n5 6\n1 6\n4 4\n",
    "general_values": "%%MatrixMarket matrix coordinate real general\n%\n% two comment lines\n4 7 6\n"
                      "1 2 0.5\n2 1 -1.25e-3\n3 7 2\n7 3 2\n4 4 1\n1 5 3.0\n",
    "rect_isolated": "%%MatrixMarket matrix coordinate integer symmetric\n9 3 3\n9 1 1\n2 3 5\n8 1 2\n",
}


def mtx_reference(text):
    L = R.lib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    libc.free.argtypes = [C.c_void_p]
    L.mtx_parse_par.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.POINTER(C.c_uint32)),
                                C.POINTER(C.POINTER(C.c_uint32))]
    L.graph_sort_edges_par.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.graph_make_simple.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.POINTER(C.c_uint32))]
    with tempfile.NamedTemporaryFile("w", suffix=".mtx", delete=False) as f:
        f.write(text)
        path = f.name
    try:
        fp = libc.fopen(path.encode(), b"r")
        N = C.c_uint32()
        Vp, Ep = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
        L.mtx_parse_par(fp, C.byref(N), C.byref(Vp), C.byref(Ep))
        libc.fclose(fp)
        L.graph_sort_edges_par(N.value, Vp, Ep)
        L.graph_make_simple(N.value, Vp, C.byref(Ep))
        n = N.value
        V = np.ctypeslib.as_array(Vp, shape=(n + 1,)).copy()
        E = np.ctypeslib.as_array(Ep, shape=(max(int(V[n]), 1),))[: int(V[n])].copy()
        libc.free(C.cast(Vp, C.c_void_p))
        libc.free(C.cast(Ep, C.c_void_p))
        return n, V, E
    finally:
        os.unlink(path)


INCIDENCE = ("incidence_degree_ordering", "saturation_degree_ordering_alt", "saturation_degree_ordering")


def incidence_golden(graphs):
    """The reference's sequential orderings (src/incidence_degree.c) and JP colors on them."""
    lib = R.lib()
    u32 = C.POINTER(C.c_uint32)
    out = {}
    for name, (N, V, E) in graphs.items():
        Vc = np.ascontiguousarray(V, np.uint32)
        Ec = np.ascontiguousarray(E if len(E) else np.zeros(1, np.uint32), np.uint32)
        for fn in INCIDENCE:
            getattr(lib, fn).argtypes = [C.c_uint32, u32, u32, C.c_void_p]
            pbuf = R.aligned(N + 8, np.float64)
            if N:
                getattr(lib, fn)(N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32), pbuf.ctypes.data)
            pv = pbuf[:N].copy()
            out[f"{name}/{fn}/p"] = pv
            out[f"{name}/{fn}/color"] = jp_color(N, V, E, pv)
    np.savez_compressed(os.path.join(OUT, "golden_incidence.npz"), **out)
    print("golden_incidence.npz", os.path.getsize(os.path.join(OUT, "golden_incidence.npz")), "bytes")


def formats_golden():
    """Texts written by the reference's writers and what its readers return for them (fast_io.c)."""
    lib = R.lib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    u32 = C.POINTER(C.c_uint32)
    out = {}
    cases = {"er300": gcn.gen_er(300, 1200, 11), "rmat9": gcn.gen_rmat(512, 8, 12), "stencil": gcn.gen_stencil27(4, 3, 3)}
    cases["edgeless"] = gcn.gen_er(12, 0, 1)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g").encode()
        for name, (N, V, E) in cases.items():
            Vc = np.ascontiguousarray(V, np.uint32)
            Ec = np.ascontiguousarray(E if len(E) else np.zeros(1, np.uint32), np.uint32)
            W = np.arange(N, dtype=np.uint32) * 3 + 1
            weighted = bool(np.all(np.diff(V.astype(np.int64)) > 0))  # the reader mis-reads weighted isolated vertices
            for store, parse in (("mtx_store", None), ("adj_store", "adj_parse"), ("gr_store", "gr_parse"),
                                 ("metis_store", "metis_parse")):
                f = libc.fopen(path, b"wb")
                if store == "metis_store":
                    getattr(lib, store).argtypes = [C.c_void_p, C.c_uint32, u32, u32, C.c_void_p]
                    getattr(lib, store)(f, N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32),
                                        W.ctypes.data if weighted else None)
                else:
                    getattr(lib, store).argtypes = [C.c_void_p, C.c_uint32, u32, u32]
                    getattr(lib, store)(f, N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32))
                libc.fclose(f)
                text = open(path, "rb").read()
                key = f"{name}/{store}"
                out[f"{key}/text"] = np.frombuffer(text, np.uint8)
                out[f"{name}/N"], out[f"{name}/V"], out[f"{name}/E"] = np.array(N), V, E
                if parse is None:
                    continue
                n, pV, pE = C.c_uint32(), u32(), u32()
                f = libc.fopen(path, b"rb")
                if parse == "metis_parse":
                    pW = u32()
                    getattr(lib, parse).argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(u32), C.POINTER(u32),
                                                    C.POINTER(u32)]
                    getattr(lib, parse)(f, C.byref(n), C.byref(pV), C.byref(pE), C.byref(pW))
                else:
                    getattr(lib, parse).argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(u32), C.POINTER(u32)]
                    getattr(lib, parse)(f, C.byref(n), C.byref(pV), C.byref(pE))
                libc.fclose(f)
                k = n.value
                rV = np.ctypeslib.as_array(pV, (k + 1,)).copy()
                rE = np.ctypeslib.as_array(pE, (max(int(rV[k]), 1),))[:int(rV[k])].copy()
                out[f"{key}/parsed_V"], out[f"{key}/parsed_E"] = rV, rE
                if parse == "metis_parse" and weighted:
                    out[f"{key}/parsed_W"] = np.ctypeslib.as_array(pW, (k,)).copy()
    np.savez_compressed(os.path.join(OUT, "golden_formats.npz"), **out)
    print("golden_formats.npz", os.path.getsize(os.path.join(OUT, "golden_formats.npz")), "bytes")


def main():
    if not R.available():
        sys.exit("oracle/_ref/libref.so is missing: run `make -C oracle` with the reference tree present")
    if "--incidence-only" in sys.argv:
        incidence_golden({**synth_graphs(), **edge_case_graphs()})
        return
    if "--formats-only" in sys.argv:
        formats_golden()
        return
    R.set_threads(4)
    synth_models = {L: gcn.synthetic_model(L, seed) for L, seed in SYNTH_MODEL_SEEDS.items()}
    ref_models = {L: gcn.model_read(os.path.join(R.MODELS, f"m{L}.gnn")) for L in (2, 3, 4)}

    graphs = {**synth_graphs(), **edge_case_graphs()}
    store = {}
    for name, (N, V, E) in graphs.items():
        store[f"{name}/N"] = np.array(N, np.int64)
        store[f"{name}/V"] = V
        store[f"{name}/E"] = E
        run_heuristics(store, name, N, V, E, synth_models)
    for L, (params, md) in synth_models.items():
        store[f"model/GNN{L}/params"] = params
        store[f"model/GNN{L}/md"] = np.array(md)
    np.savez_compressed(os.path.join(OUT, "golden_synth.npz"), **store)

    ref = {}
    for name in ("er1500", "rmat11", "bridged"):
        N, V, E = graphs[name]
        for L, (params, md) in ref_models.items():
            p = R.graph_sage(params, md, N, V, E)
            ref[f"{name}/GNN{L}/p"] = p
            ref[f"{name}/GNN{L}/color"] = jp_color(N, V, E, p)
    np.savez_compressed(os.path.join(OUT, "golden_refmodels.npz"), **ref)

    mtx = {}
    for name, text in MTX_CASES.items():
        n, V, E = mtx_reference(text)
        mtx[f"{name}/text"] = np.frombuffer(text.encode(), np.uint8)
        mtx[f"{name}/N"] = np.array(n)
        mtx[f"{name}/V"] = V
        mtx[f"{name}/E"] = E
    np.savez_compressed(os.path.join(OUT, "golden_mtx.npz"), **mtx)
    for f in ("golden_synth.npz", "golden_refmodels.npz", "golden_mtx.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")
    incidence_golden(graphs)
    formats_golden()


if __name__ == "__main__":
    main()
