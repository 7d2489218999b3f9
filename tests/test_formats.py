"""The reference's other graph formats (src/fast_io.c:224-437), host code of the library: the
writers print the reference's text byte for byte, the readers return the reference's V, E (and
METIS weights), and gc_read_graph turns any of them into the simple, sorted CSR of the MTX path."""
import ctypes as C
import os

import numpy as np
import pytest

import gnn_coloring as gcn
from conftest import GOLDEN

u32 = C.POINTER(C.c_uint32)
libc = C.CDLL(None)
libc.fopen.restype = C.c_void_p
libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
libc.fclose.argtypes = [C.c_void_p]
STORES = ("mtx_store", "adj_store", "gr_store", "metis_store")
PARSES = {"adj_store": "adj_parse", "gr_store": "gr_parse", "metis_store": "metis_parse"}


def store(lib, fn, path, N, V, E, W=None):
    Vc = np.ascontiguousarray(V, np.uint32)
    Ec = np.ascontiguousarray(E if len(E) else np.zeros(1, np.uint32), np.uint32)
    f = libc.fopen(str(path).encode(), b"wb")
    if fn == "metis_store":
        getattr(lib, fn).argtypes = [C.c_void_p, C.c_uint32, u32, u32, C.c_void_p]
        getattr(lib, fn)(f, N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32), None if W is None else W.ctypes.data)
    else:
        getattr(lib, fn).argtypes = [C.c_void_p, C.c_uint32, u32, u32]
        getattr(lib, fn)(f, N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32))
    libc.fclose(f)
    return open(path, "rb").read()


def parse(lib, fn, path):
    n, pV, pE, pW = C.c_uint32(), u32(), u32(), u32()
    f = libc.fopen(str(path).encode(), b"rb")
    if fn == "metis_parse":
        getattr(lib, fn).argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
        getattr(lib, fn)(f, C.byref(n), C.byref(pV), C.byref(pE), C.byref(pW))
    else:
        getattr(lib, fn).argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(u32), C.POINTER(u32)]
        getattr(lib, fn)(f, C.byref(n), C.byref(pV), C.byref(pE))
    libc.fclose(f)
    k = n.value
    V = np.ctypeslib.as_array(pV, (k + 1,)).copy()
    E = np.ctypeslib.as_array(pE, (max(int(V[k]), 1),))[:int(V[k])].copy()
    W = np.ctypeslib.as_array(pW, (k,)).copy() if (fn == "metis_parse" and pW) else None
    return k, V, E, W


def test_formats_match_golden(tmp_path):
    z = np.load(os.path.join(GOLDEN, "golden_formats.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    for name in names:
        N, V, E = int(z[f"{name}/N"]), z[f"{name}/V"], z[f"{name}/E"]
        weighted = f"{name}/metis_store/parsed_W" in z.files
        W = np.arange(N, dtype=np.uint32) * 3 + 1
        for fn in STORES:
            text = store(gcn.lib, fn, tmp_path / fn, N, V, E, W if (fn == "metis_store" and weighted) else None)
            assert text == z[f"{name}/{fn}/text"].tobytes(), (name, fn)
            if fn in PARSES:
                path = tmp_path / (fn + ".in")
                path.write_bytes(z[f"{name}/{fn}/text"].tobytes())
                k, pV, pE, pW = parse(gcn.lib, PARSES[fn], path)
                assert k == N and np.array_equal(pV, z[f"{name}/{fn}/parsed_V"]), (name, fn)
                assert np.array_equal(pE, z[f"{name}/{fn}/parsed_E"]), (name, fn)
                if weighted and fn == "metis_store":
                    assert np.array_equal(pW, z[f"{name}/{fn}/parsed_W"])


def test_hand_written_files_match_reference(tmp_path):
    from oracle import reference as R
    if not R.available():
        pytest.skip("the reference was not compiled here (oracle/_ref)")
    L = R.lib()
    files = {"m.graph": "% comment\n4 4 11\n5 2 9 3 1 \n6 1 9\n7 1 1 4 2  \n8 3 2\n",
             "n.graph": "3 2 0\n2 3\n1\n1\n",
             "p.gr": "c hello\nc more\np td 5 4\n1 2\nc mid\n2 3\n3 3\n5 1\n",
             "a.adj": "AdjacencyGraph\n3\n4\n0\n2\n3\n1\n2\n0\n0\n"}
    for fname, text in files.items():
        path = tmp_path / fname
        path.write_text(text)
        fn = {"graph": "metis_parse", "gr": "gr_parse", "adj": "adj_parse"}[fname.split(".")[1]]
        r, o = parse(L, fn, path), parse(gcn.lib, fn, path)
        assert r[0] == o[0] and np.array_equal(r[1], o[1]) and np.array_equal(r[2], o[2]), fname
        assert (r[3] is None) == (o[3] is None) and (r[3] is None or np.array_equal(r[3], o[3])), fname


def test_read_graph_any_format(tmp_path):
    N, V, E = gcn.gen_rmat(1 << 10, 8, 7)
    fns = {".mtx": "mtx_store", ".adj": "adj_store", ".gr": "gr_store", ".graph": "metis_store"}
    for ext, fn in fns.items():
        path = tmp_path / ("g" + ext)
        store(gcn.lib, fn, path, N, V, E)
        n, pV, pE = C.c_uint32(), u32(), u32()
        gcn.lib.gc_read_graph.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(u32), C.POINTER(u32)]
        assert gcn.lib.gc_read_graph(str(path).encode(), C.byref(n), C.byref(pV), C.byref(pE)) == 0, ext
        k = n.value
        rV = np.ctypeslib.as_array(pV, (k + 1,)).copy()
        rE = np.ctypeslib.as_array(pE, (max(int(rV[k]), 1),))[:int(rV[k])].copy()
        assert k == N and np.array_equal(rV, V) and np.array_equal(rE, E), ext
    bad = tmp_path / "g.xyz"
    bad.write_text("1 2\n")
    assert gcn.lib.gc_read_graph(str(bad).encode(), C.byref(C.c_uint32()), C.byref(u32()), C.byref(u32())) == 6
