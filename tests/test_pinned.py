"""Uploads and downloads from page-locked host memory take the overlapped paths: E goes up on a copy
stream while the graph is prepared from V, and the reference-facing X_internal_par calls bring the
priorities down while the coloring runs.  Results must equal those from pageable memory and the
golden vectors, and malformed CSRs must still be refused."""
import ctypes as C

import numpy as np
import pytest

import gnn_coloring as gcn

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def pinned_copy(a, dtype):
    a = np.ascontiguousarray(a, dtype)
    t = torch.empty(max(len(a), 1), dtype={np.uint32: torch.int32, np.float64: torch.float64,
                                           np.int32: torch.int32}[dtype]).pin_memory()
    view = t.numpy().view(dtype)[: len(a)]
    view[:] = a
    return t, view


def test_pinned_upload_matches_pageable(gpu_ctx, golden):
    model = gcn.Model(gpu_ctx, *golden.model(3))
    graphs = [(name, golden.graph(name)) for name in ("er1500", "rmat11", "bridged", "path7")]
    graphs.append(("rmat16", gcn.gen_rmat(1 << 16, 16, 4)))
    for name, (N, V, E) in graphs:
        keep_v, pV = pinned_copy(V, np.uint32)
        keep_e, pE = pinned_copy(E, np.uint32)
        for heur in ("LF", "GNN"):
            gp = gcn.Graph(gpu_ctx, N, pV, pE)
            gh = gcn.Graph(gpu_ctx, N, V, E)
            for g in (gp, gh):
                g.priority(heur, model if heur == "GNN" else None)
            assert gp.color(recolor=1) == gh.color(recolor=1), (name, heur)
            assert np.array_equal(gp.colors(), gh.colors()), (name, heur)
            assert np.array_equal(gp.priorities(), gh.priorities()), (name, heur)
            gp.close()
            gh.close()
        if name in ("er1500", "rmat11", "bridged", "path7"):
            g = gcn.Graph(gpu_ctx, N, pV, pE)
            g.priority("GNN", model)
            assert np.array_equal(g.priorities(), golden.get(name, "GNN3", "p")), name
            g.close()
        del keep_v, keep_e


def test_pinned_malformed_csr_is_refused(gpu_ctx):
    N, V, E = gcn.gen_er(2000, 8000, 3)
    _, pV = pinned_copy(V, np.uint32)
    keep, pE = pinned_copy(E, np.uint32)
    pE[17] = N + 5  # an id outside the graph
    with pytest.raises(gcn.GCError) as e:
        gcn.Graph(gpu_ctx, N, pV, pE)
    assert e.value.name == "GC_ERR_INVALID"
    _, pV2 = pinned_copy(V, np.uint32)
    pV2[10] = pV2[12] + 1  # offsets not monotone
    _, pE2 = pinned_copy(E, np.uint32)
    with pytest.raises(gcn.GCError) as e:
        gcn.Graph(gpu_ctx, N, pV2, pE2)
    assert e.value.name == "GC_ERR_INVALID"
    # the context stays usable
    g = gcn.Graph(gpu_ctx, N, pV, np.ascontiguousarray(E, np.uint32))
    h = gcn.Graph(gpu_ctx, N, V, E)
    g.priority("LF")
    h.priority("LF")
    assert g.color() == h.color()
    del keep


def test_legacy_internal_par_from_pinned_buffers(golden, tmp_path, monkeypatch):
    """gnn_internal_par with page-locked V, E, p and color: the priorities (downloaded beside the
    coloring) and the colors equal the golden vectors, twice in a row."""
    params, md = golden.model(3)
    gcn.model_write(str(tmp_path / "m3.gnn"), params, md)
    monkeypatch.setenv("GC_MODEL_DIR", str(tmp_path))
    lib = gcn.lib
    C.c_int.in_dll(lib, "layers").value = 3
    lib.gnn_setup.argtypes = [C.c_uint32, C.c_uint32]
    lib.gnn_setup.restype = C.c_void_p
    lib.jones_plassmann_setup.argtypes = [C.c_uint32, C.c_uint32]
    lib.jones_plassmann_setup.restype = C.c_void_p
    lib.gnn_internal_par.argtypes = [C.c_uint32] + [C.c_void_p] * 6
    lib.gnn_cleanup.argtypes = [C.c_void_p]
    lib.jones_plassmann_cleanup.argtypes = [C.c_void_p]
    for name in ("er1500", "rmat11"):
        N, V, E = golden.graph(name)
        tv, _ = pinned_copy(V, np.uint32)
        te, _ = pinned_copy(E, np.uint32)
        tp = torch.empty(N + 8, dtype=torch.float64).pin_memory()
        tc = torch.empty(N, dtype=torch.int32).pin_memory()
        ad = lib.gnn_setup(N, int(V[N]))
        jp = lib.jones_plassmann_setup(N, int(V[N]))
        for _ in range(2):
            tp.zero_()
            tc.zero_()
            lib.gnn_internal_par(N, tv.data_ptr(), te.data_ptr(), ad, jp, tp.data_ptr(), tc.data_ptr())
            assert np.array_equal(tp.numpy()[:N], golden.get(name, "GNN3", "p")), name
            assert np.array_equal(tc.numpy(), golden.get(name, "GNN3", "color")), name
        lib.gnn_cleanup(ad)
        lib.jones_plassmann_cleanup(jp)


def test_gnn_rows_built_while_pinned_e_arrives(gpu_ctx, golden):
    """With GNN priorities announced (gc_graph_gnn_hint, what the reference-named GNN calls do), a
    page-locked E goes up in pieces and each piece is turned into feature rows as it arrives; that
    conversion also checks the ids.  An id outside the graph in the first, a middle or the last piece
    is refused, the graph then takes a good upload, and GNN3 priorities, LF colors and Culberson
    rounds equal those of a plain upload."""
    lib = gcn.lib
    lib.gc_graph_gnn_hint.argtypes = [C.c_void_p, C.c_int]
    lib.gc_graph_gnn_hint.restype = None
    model = gcn.Model(gpu_ctx, *golden.model(3))
    for name in ("rmat11", "er1500"):
        N, V, E = golden.graph(name)
        M = len(E)
        h = C.c_void_p()
        gpu_ctx.check(lib.gc_graph_create(gpu_ctx.h, N, M, C.byref(h)), "create")
        lib.gc_graph_gnn_hint(h, 1)
        keep_v, pV = pinned_copy(V, np.uint32)
        keep_e, pE = pinned_copy(E, np.uint32)
        vp_, ep_ = pV.ctypes.data_as(C.POINTER(C.c_uint32)), pE.ctypes.data_as(C.POINTER(C.c_uint32))
        for bad in (3, M // 2, M - 1):
            pE[bad] = N + 7
            assert lib.gc_graph_reupload(gpu_ctx.h, h, N, vp_, ep_) == 1, (name, bad)  # GC_ERR_INVALID
            pE[bad] = E[bad]
        assert lib.gc_graph_reupload(gpu_ctx.h, h, N, vp_, ep_) == 0, name
        ref = gcn.Graph(gpu_ctx, N, V, E)
        assert lib.gc_priority(gpu_ctx.h, h, gcn.GC_GNN, model.h) == 0
        p = np.empty(N, np.float64)
        assert lib.gc_download_priority(gpu_ctx.h, h, p.ctypes.data_as(C.POINTER(C.c_double))) == 0
        assert np.array_equal(p, golden.get(name, "GNN3", "p")), name
        # the rows built at upload do not disturb the other heuristics
        assert lib.gc_priority(gpu_ctx.h, h, gcn.GC_LF, None) == 0
        ref.priority("LF")
        used = C.c_int()
        assert lib.gc_color(gpu_ctx.h, h, 1, C.byref(used)) == 0
        assert used.value == ref.color(recolor=1), name
        ref.close()
        lib.gc_graph_free(h)
        del keep_v, keep_e
