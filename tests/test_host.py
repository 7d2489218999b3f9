"""Host-side graph preparation: Matrix Market rules, generators, .gnn models (no GPU)."""
import os

import numpy as np
import pytest

import gnn_coloring as gcn


def is_simple_sorted_symmetric(N, V, E):
    if V[0] != 0 or np.any(np.diff(V.astype(np.int64)) < 0) or V[N] != len(E):
        return False
    edges = set()
    for u in range(N):
        row = E[V[u]:V[u + 1]]
        if np.any(np.diff(row.astype(np.int64)) <= 0) or np.any(row == u) or np.any(row >= N):
            return False
        edges.update((u, int(v)) for v in row)
    return all((v, u) in edges for (u, v) in edges)


def test_mtx_matches_reference_csr(golden_mtx, tmp_path):
    names = sorted({k.split("/")[0] for k in golden_mtx.files})
    for name in names:
        path = tmp_path / f"{name}.mtx"
        path.write_bytes(golden_mtx[f"{name}/text"].tobytes())
        N, V, E = gcn.mtx_read(str(path))
        assert N == int(golden_mtx[f"{name}/N"]), name
        assert np.array_equal(V, golden_mtx[f"{name}/V"]), name
        assert np.array_equal(E, golden_mtx[f"{name}/E"]), name


def test_mtx_rejects_bad_indices(tmp_path):
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n1 2\n0 3\n")
    with pytest.raises(gcn.GCError) as e:
        gcn.mtx_read(str(bad))
    assert e.value.name == "GC_ERR_FORMAT"
    trunc = tmp_path / "trunc.mtx"
    trunc.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 5\n1 2\n")
    with pytest.raises(gcn.GCError):
        gcn.mtx_read(str(trunc))
    with pytest.raises(gcn.GCError) as e:
        gcn.mtx_read(str(tmp_path / "missing.mtx"))
    assert e.value.name == "GC_ERR_IO"


def test_mtx_roundtrip(tmp_path):
    N, V, E = gcn.gen_rmat(1 << 10, 8, 5)
    path = str(tmp_path / "g.mtx")
    gcn.mtx_write(path, N, V, E)
    N2, V2, E2 = gcn.mtx_read(path)
    assert N2 == N and np.array_equal(V, V2) and np.array_equal(E, E2)


def test_generators_deterministic_and_simple():
    a = gcn.gen_er(3000, 20000, 5)
    b = gcn.gen_er(3000, 20000, 5)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert a[1][-1] == 40000  # exactly m undirected edges
    assert is_simple_sorted_symmetric(*a)
    r = gcn.gen_rmat(1 << 12, 8, 9)
    assert is_simple_sorted_symmetric(*r)
    g = gcn.gen_rgg2d(4000, 0.03, 1)
    assert is_simple_sorted_symmetric(*g)
    s = gcn.gen_stencil27(5, 4, 3)
    assert is_simple_sorted_symmetric(*s)
    # interior vertices of a 27-point stencil have 26 neighbours; M = prod(3n-2) - prod(n)
    assert s[1][-1] == (13 * 10 * 7) - (5 * 4 * 3)


def test_generators_match_golden_graphs(golden):
    """The committed fixtures were made on these generators: they must not drift."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", os.path.join(os.path.dirname(__file__), "golden",
                                                                     "make_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    for name, (N, V, E) in {**mk.synth_graphs(), **mk.edge_case_graphs()}.items():
        n2, V2, E2 = golden.graph(name)
        assert N == n2 and np.array_equal(V, V2) and np.array_equal(E, E2), name
    for L, seed in mk.SYNTH_MODEL_SEEDS.items():
        params, md = gcn.synthetic_model(L, seed)
        gp, gmd = golden.model(L)
        assert np.array_equal(params, gp) and md == gmd


def test_rmat_non_power_of_two_rejects_out_of_range():
    N, V, E = gcn.gen_rmat(1000, 8, 4)
    assert N == 1000 and (len(E) == 0 or E.max() < 1000)
    assert is_simple_sorted_symmetric(N, V, E)


def test_model_roundtrip(tmp_path):
    for L in (2, 3, 4):
        params, md = gcn.synthetic_model(L, 40 + L)
        path = str(tmp_path / f"m{L}.gnn")
        gcn.model_write(path, params, md)
        p2, md2 = gcn.model_read(path)
        assert md2 == md and np.array_equal(p2, params)


def test_model_format_errors(tmp_path):
    bad = tmp_path / "bad.gnn"
    bad.write_text("100 5\n1 2 3\n")  # fewer than 2 layers
    with pytest.raises(gcn.GCError):
        gcn.model_read(str(bad))
    short = tmp_path / "short.gnn"
    short.write_text("1056 100\n" + " ".join(["0.5"] * 100))
    with pytest.raises(gcn.GCError):
        gcn.model_read(str(short))


# ---- the reference's sequential orderings (host code of the library) -------------------------------

INCIDENCE = ("incidence_degree_ordering", "saturation_degree_ordering_alt", "saturation_degree_ordering")


def _ordering(fn, N, V, E):
    import ctypes as C
    u32 = C.POINTER(C.c_uint32)
    f = getattr(gcn.lib, fn)
    f.argtypes = [C.c_uint32, u32, u32, C.c_void_p]
    Vc = np.ascontiguousarray(V, np.uint32)
    Ec = np.ascontiguousarray(E if len(E) else np.zeros(1, np.uint32), np.uint32)
    p = np.zeros(N + 8)
    if N:
        f(N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32), p.ctypes.data)
    return p[:N]


def test_incidence_orderings_match_golden(golden):
    """ID, SDA and SD priorities equal the reference's (golden vectors from src/incidence_degree.c),
    including components reached late and a last vertex that the reference never orders (p = -1)."""
    inc = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_incidence.npz"))
    for name in golden.graphs:
        N, V, E = golden.graph(name)
        for fn in INCIDENCE:
            assert np.array_equal(_ordering(fn, N, V, E), inc[f"{name}/{fn}/p"]), (name, fn)


def test_incidence_orderings_match_live_reference():
    from oracle import reference as R
    if not R.available():
        pytest.skip("the reference was not compiled here (oracle/_ref)")
    import ctypes as C
    L = R.lib()
    u32 = C.POINTER(C.c_uint32)
    pairs_n = 60
    I = np.array([0, 1, 2, 10, 11, 20, 21, 22, 30, 31], np.uint32)
    J = np.array([1, 2, 0, 11, 12, 21, 22, 20, 31, 58], np.uint32)
    graphs = [gcn.gen_er(3000, 20000, 5), gcn.gen_rmat(1 << 12, 8, 3), gcn.gen_rmat(5000, 4, 9),
              gcn.gen_stencil27(9, 8, 7), gcn.csr_from_pairs(pairs_n, I, J), gcn.gen_er(40, 0, 1)]
    for N, V, E in graphs:
        Vc = np.ascontiguousarray(V, np.uint32)
        Ec = np.ascontiguousarray(E if len(E) else np.zeros(1, np.uint32), np.uint32)
        for fn in INCIDENCE:
            getattr(L, fn).argtypes = [C.c_uint32, u32, u32, C.c_void_p]
            ref = R.aligned(N + 8, np.float64)
            getattr(L, fn)(N, Vc.ctypes.data_as(u32), Ec.ctypes.data_as(u32), ref.ctypes.data)
            assert np.array_equal(_ordering(fn, N, V, E), ref[:N]), (N, fn)


def test_numpy_rmat_samples_give_the_library_graph():
    """The reference arm of bench.py builds its graph without the library: synthgen's numpy R-MAT
    samples, turned into a CSR by the reference's own mtx_to_graph_par + graph_sort_edges_par +
    graph_make_simple.  That CSR must be the library's gen_rmat graph exactly."""
    import synthgen
    from oracle import reference as R
    if not R.available():
        pytest.skip("oracle/_ref/libref.so not built")
    for scale, seed, ef in ((10, 2, 16), (13, 7, 16), (12, 5, 8.5)):
        n = 1 << scale
        I, J = synthgen.rmat_samples(n, ef, seed, workers=1)
        V, E = R.csr_from_samples(n, I, J)
        _, V2, E2 = gcn.gen_rmat(n, ef, seed)
        assert np.array_equal(V, V2) and np.array_equal(E, E2), (scale, seed)
    # non-power-of-two n: samples with an id >= n are dropped, as the library does
    I, J = synthgen.rmat_samples(3000, 8, 11, workers=1)
    V, E = R.csr_from_samples(3000, I, J)
    _, V2, E2 = gcn.gen_rmat(3000, 8, 11)
    assert np.array_equal(V, V2) and np.array_equal(E, E2)
