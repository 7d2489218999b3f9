"""Batches of independent graphs (gc_batch_*): every graph's priorities, colors and color count in a
batch must equal the same graph colored alone -- by the plain device path and by the oracle.

CPU tests cover the mixed-graph generator rule and the host-side helpers; GPU tests call the
library's batch entry points through the C ABI."""
import numpy as np
import pytest

import gnn_coloring as gcn

ORACLE_MD = 100


def _oracle():
    from oracle import restatement as orc
    return orc


def _small_mixed(G, seed0, n_min=40, n_max=3000):
    return [gcn.gen_mixed(seed0 + i, n_min, n_max)[:3] for i in range(G)]


def _edge_cases():
    """Graphs the mixed generator never makes: empty, edgeless, a single edge, a star, a clique."""
    star_n = 70
    sV = np.concatenate([[0, star_n - 1], np.arange(star_n, 2 * star_n - 1)]).astype(np.uint32)
    sE = np.concatenate([np.arange(1, star_n), np.zeros(star_n - 1)]).astype(np.uint32)
    k = 9
    kV = (np.arange(k + 1) * (k - 1)).astype(np.uint32)
    kE = np.array([v for u in range(k) for v in range(k) if v != u], np.uint32)
    return [
        (0, np.zeros(1, np.uint32), np.zeros(0, np.uint32)),
        (5, np.zeros(6, np.uint32), np.zeros(0, np.uint32)),
        (2, np.array([0, 1, 2], np.uint32), np.array([1, 0], np.uint32)),
        (star_n, sV, sE),
        (k, kV, kE),
        (1, np.zeros(2, np.uint32), np.zeros(0, np.uint32)),
    ]


# ---- host side (no GPU) --------------------------------------------------------------------------

def test_mixed_generator_rule():
    for seed in range(1000, 1012):
        N, V, E, kind, param = gcn.gen_mixed(seed, 1000, 200000)
        assert 1000 <= N <= 200000
        assert kind == seed % 2
        if kind == 0:
            assert 8.0 <= param <= 32.0
            assert len(E) == 2 * round(N * param / 2)  # G(n, m): m distinct pairs, both directions
        else:
            assert param == 8.0 and len(E) <= 16 * N
        d = np.diff(V.astype(np.int64))
        assert d.min() >= 0 and V[-1] == len(E)
        # simple and symmetric
        src = np.repeat(np.arange(N), d)
        assert not np.any(src == E)
        fwd = set(zip(src.tolist(), E.tolist()))
        assert all((v, u) in fwd for u, v in list(fwd)[:2000])
    # the same seed gives the same graph
    a, b = gcn.gen_mixed(1234), gcn.gen_mixed(1234)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_mixed_batch_is_concatenation():
    G = 10
    voff, V, E = gcn.gen_mixed_batch(G, 77, 100, 5000)
    assert voff[0] == 0 and len(voff) == G + 1 and V[-1] == len(E)
    for g in range(G):
        N, Vg, Eg = gcn.split_batch(voff, V, E, g)
        N2, V2, E2, _, _ = gcn.gen_mixed(77 + g, 100, 5000)
        assert N == N2 and np.array_equal(Vg, V2) and np.array_equal(Eg, E2)


def test_device_bytes_model():
    small = gcn.batch_device_bytes(1, 1000, 16000, "LF")
    gnn = gcn.batch_device_bytes(1, 1000, 16000, "GNN")
    assert gnn > small > 8 * 16000
    # the full 4,096-graph mix (N ~ 1.5e8, M ~ 2.5e9) fits a 180 GB B200 with room to spare
    assert gcn.batch_device_bytes(4096, 150_000_000, 2_500_000_000, "GNN") < 90e9


# ---- device ------------------------------------------------------------------------------------

@pytest.fixture(scope="module")
def models(gpu_ctx):
    return {L: gcn.Model(gpu_ctx, *gcn.synthetic_model(L, 1000 + L, ORACLE_MD)) for L in (2, 3, 4)}


def _plain(ctx, graph, heur, model, recolor=0):
    N, V, E = graph
    g = gcn.Graph(ctx, N, V, E)
    g.priority(heur, model)
    c = g.color(recolor)
    col, p = g.colors(), g.priorities()
    g.close()
    return col, c, p


def _check_batch_against_plain(ctx, graphs, heur, model=None, recolor=0, tuning=None):
    b = gcn.Batch(ctx, graphs=graphs)
    if tuning is not None:
        b.tuning = tuning
    counts = b.color(heur, model, recolor)
    allc = b.colors()
    allp = b.priorities()
    for i, graph in enumerate(graphs):
        col, c, p = _plain(ctx, graph, heur, model, recolor)
        got = b.graph_colors(i, allc)
        assert np.array_equal(got, col), f"graph {i}: colors differ from the plain path"
        assert counts[i] == c, f"graph {i}: color count {counts[i]} != {c}"
        if recolor == 0:
            a, z = int(b.voff[i]), int(b.voff[i + 1])
            assert np.array_equal(allp[a:z], p), f"graph {i}: priorities differ"
    b.close()
    return counts


@pytest.mark.gpu
@pytest.mark.parametrize("heur", ["FF", "LF", "LLF", "GNN2", "GNN3"])
def test_batch_matches_oracle(gpu_ctx, models, heur):
    orc = _oracle()
    graphs = _small_mixed(12, 5000) + _edge_cases()
    h, L = ("GNN", int(heur[3])) if heur.startswith("GNN") else (heur, 0)
    model = models[L] if L else None
    b = gcn.Batch(gpu_ctx, graphs=graphs)
    counts = b.color(h, model)
    allc = b.colors()
    for i, (N, V, E) in enumerate(graphs):
        if L:
            params, md = gcn.synthetic_model(L, 1000 + L, ORACLE_MD)
            p = orc.ordering("GNN", N, V, E, params, md)
        else:
            p = orc.ordering(heur, N, V, E)
        want, _ = orc.greedy_color(N, V, E, p)
        assert np.array_equal(b.graph_colors(i, allc), want), f"graph {i} ({heur})"
        assert counts[i] == orc.validate(N, V, E, want)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("heur", ["FF", "LLF", "GNN3"])
def test_batch_matches_plain_path(gpu_ctx, models, heur):
    graphs = _small_mixed(16, 6100, 200, 20000) + _edge_cases()
    h, L = ("GNN", 3) if heur == "GNN3" else (heur, 0)
    _check_batch_against_plain(gpu_ctx, graphs, h, models[3] if L else None)


@pytest.mark.gpu
def test_batch_culberson(gpu_ctx, models):
    orc = _oracle()
    graphs = _small_mixed(8, 7000, 100, 4000)
    b = gcn.Batch(gpu_ctx, graphs=graphs)
    counts = b.color("GNN", models[4], recolor=3)
    allc = b.colors()
    params, md = gcn.synthetic_model(4, 1004, ORACLE_MD)
    for i, (N, V, E) in enumerate(graphs):
        first, _ = orc.greedy_color(N, V, E, orc.ordering("GNN", N, V, E, params, md))
        want = orc.culberson(N, V, E, first, 3)
        assert np.array_equal(b.graph_colors(i, allc), want)
        assert counts[i] == orc.validate(N, V, E, want) <= orc.validate(N, V, E, first)
    b.close()


@pytest.mark.gpu
def test_captured_replays_repeat(gpu_ctx, models):
    graphs = _small_mixed(20, 8000, 100, 30000)
    b = gcn.Batch(gpu_ctx, graphs=graphs)
    l0 = gpu_ctx.launches
    first = b.color("GNN", models[2])      # direct pass, then capture
    c1 = b.colors()
    l1 = gpu_ctx.launches
    for _ in range(3):
        again = b.color("GNN", models[2])  # graph replays
        assert np.array_equal(again, first)
        assert np.array_equal(b.colors(), c1)
    per_replay = (gpu_ctx.launches - l1) / 3
    assert 0 < per_replay <= l1 - l0
    # another heuristic on the same batch, then back
    lf = b.color("LF")
    assert np.array_equal(b.color("GNN", models[2]), first)
    assert np.array_equal(b.color("LF"), lf)
    b.close()


@pytest.mark.gpu
def test_tunings_do_not_change_results(gpu_ctx, models):
    graphs = _small_mixed(10, 9000, 300, 60000)
    base = _check_batch_against_plain(gpu_ctx, graphs, "GNN", models[3])
    variants = []
    for sched in (gcn.GC_SCHEDULE_DEGREE, gcn.GC_SCHEDULE_SEGMENT):
        for warp, hub, ctas, tight, nap, gwarp in ((0, 16, 1, 4, 8, 8), (16, 64, 4, 128, 32, 64),
                                                  (1024, 4096, 3, 32, 128, 4096)):
            t = gcn.default_tuning()
            t.schedule, t.warp_degree, t.hub_degree = sched, warp, hub
            t.jp_ctas_per_sm, t.jp_tight, t.jp_nap = ctas, tight, nap
            t.gnn_warp_degree = gwarp
            variants.append(t)
    for t in variants:
        counts = _check_batch_against_plain(gpu_ctx, graphs, "GNN", models[3], tuning=t)
        assert np.array_equal(counts, base)


@pytest.mark.gpu
def test_autotune_keeps_results(gpu_ctx, models):
    graphs = _small_mixed(24, 9500, 100, 20000)
    b = gcn.Batch(gpu_ctx, graphs=graphs)
    before = b.color("GNN", models[2])
    cols = b.colors()
    t, ms = b.autotune("GNN", models[2], effort=1)
    assert ms > 0
    assert b.tuning.as_dict() == t.as_dict()
    assert np.array_equal(b.color("GNN", models[2]), before)
    assert np.array_equal(b.colors(), cols)
    b.close()


@pytest.mark.gpu
def test_flat_upload_and_reupload(gpu_ctx, models):
    voff, V, E = gcn.gen_mixed_batch(9, 4242, 50, 8000)
    flat = gcn.Batch(gpu_ctx, voff, V, E)
    graphs = [gcn.split_batch(voff, V, E, g) for g in range(9)]
    listed = gcn.Batch(gpu_ctx, graphs=graphs)
    assert flat.N == listed.N == int(voff[-1]) and flat.M == listed.M == len(E)
    a = flat.color("GNN", models[3])
    b = listed.color("GNN", models[3])
    assert np.array_equal(a, b) and np.array_equal(flat.colors(), listed.colors())
    # refill an allocated batch with other graphs, then with the first ones again
    other = _small_mixed(5, 4300, 50, 3000)
    ns = np.array([n for n, _, _ in other], np.uint32)
    import ctypes as C
    keep = [(np.ascontiguousarray(v, np.uint32), np.ascontiguousarray(e, np.uint32)) for _, v, e in other]
    Vs = (gcn.u32p * len(keep))(*[gcn._ptr(v, gcn.u32p) for v, _ in keep])
    Es = (gcn.u32p * len(keep))(*[gcn._ptr(e, gcn.u32p) for _, e in keep])
    gpu_ctx.check(gcn.lib.gc_batch_reupload_graphs(gpu_ctx.h, flat.h, len(other), gcn._ptr(ns, gcn.u32p), Vs, Es))
    flat.voff = np.concatenate([[0], np.cumsum(ns)]).astype(np.uint32)
    flat.G = len(other)
    got = flat.color("LF")
    ref = gcn.Batch(gpu_ctx, graphs=other)
    assert np.array_equal(got, ref.color("LF")) and np.array_equal(flat.colors(), ref.colors())
    flat.close(), listed.close(), ref.close()


@pytest.mark.gpu
def test_batch_rejects_bad_input(gpu_ctx, models):
    graphs = _small_mixed(3, 100, 50, 500)
    b = gcn.Batch(gpu_ctx, graphs=graphs)
    for heur in ("SL", "SLL"):
        with pytest.raises(gcn.GCError) as e:
            b.color(heur)
        assert e.value.status == 1
    with pytest.raises(gcn.GCError):
        b.color("GNN", None)
    b.close()
    # a neighbour id outside its own graph
    N, V, E = graphs[0]
    E2 = E.copy()
    E2[0] = N + 3
    with pytest.raises(gcn.GCError) as e:
        gcn.Batch(gpu_ctx, graphs=[graphs[1], (N, V, E2)])
    assert e.value.status == 1
    # row offsets that run backwards
    V3 = V.copy()
    V3[1], V3[2] = V3[2], V3[1]
    if V3[1] != V3[2]:
        with pytest.raises(gcn.GCError):
            gcn.Batch(gpu_ctx, graphs=[(N, V3, E)])
    # the context stays usable
    ok = gcn.Batch(gpu_ctx, graphs=graphs)
    assert (ok.color("FF") > 0).all()
    ok.close()


@pytest.mark.gpu
def test_reupload_from_device_graphs(gpu_ctx, models):
    """gc_batch_reupload_device_graphs: a batch gathered from device-resident CSRs colors exactly like
    the same graphs uploaded from host memory."""
    import ctypes as C
    import torch
    graphs = _small_mixed(9, 600) + _edge_cases()
    dev = [(torch.from_numpy(V.astype(np.int32)).cuda(), torch.from_numpy(E.astype(np.int32) if len(E) else
                                                                           np.zeros(1, np.int32)).cuda())
           for _, V, E in graphs]
    torch.cuda.synchronize()
    G = len(graphs)
    b = gcn.Batch(gpu_ctx, graphs=graphs)
    ref_counts = b.color("GNN", models[3])
    ref = b.colors()
    bh = C.c_void_p()
    gpu_ctx.check(gcn.lib.gc_batch_create(gpu_ctx.h, G + 3, b.N + 10, b.M + 10, C.byref(bh)), "create")
    n = np.array([g[0] for g in graphs], np.uint32)
    m = np.array([int(g[1][-1]) for g in graphs], np.uint32)
    u32p = C.POINTER(C.c_uint32)
    dVs = (u32p * G)(*[C.cast(v.data_ptr(), u32p) for v, _ in dev])
    dEs = (u32p * G)(*[C.cast(e.data_ptr(), u32p) for _, e in dev])
    for _ in range(2):  # twice: the second refill reuses the first one's buffers
        gpu_ctx.check(gcn.lib.gc_batch_reupload_device_graphs(gpu_ctx.h, bh, G, n.ctypes.data_as(u32p),
                                                              m.ctypes.data_as(u32p), dVs, dEs), "refill")
        counts = np.zeros(G, np.int32)
        gpu_ctx.check(gcn.lib.gc_batch_color_once(gpu_ctx.h, bh, gcn.GC_GNN, models[3].h, 0,
                                                  counts.ctypes.data_as(C.POINTER(C.c_int32))), "color")
        got = np.zeros(max(b.N, 1), np.int32)
        gpu_ctx.check(gcn.lib.gc_batch_download_colors(gpu_ctx.h, bh, got.ctypes.data_as(C.POINTER(C.c_int32))),
                      "colors")
        assert np.array_equal(counts, ref_counts)
        assert np.array_equal(got[: b.N], ref)
    gcn.lib.gc_batch_free(bh)
    b.close()
