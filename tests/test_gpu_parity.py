"""GPU parity: the CUDA path (through the C ABI) against the reference's golden vectors and the
oracle.  Integer heuristics and colors must be identical; GraphSAGE priorities must be identical
bit for bit (tolerance 0: the kernels reproduce the reference's FP32 operation order)."""
import os
import subprocess

import numpy as np
import pytest

import gnn_coloring as gcn
from conftest import GOLDEN, HEURISTICS, PKG
from oracle import reference as R
from oracle import restatement as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models(gpu_ctx, golden):
    return {L: gcn.Model(gpu_ctx, *golden.model(L)) for L in (2, 3, 4)}


def gpu_run(ctx, N, V, E, heur, models):
    g = gcn.Graph(ctx, N, V, E)
    if heur.startswith("GNN"):
        g.priority("GNN", models[int(heur[3:])])
    else:
        g.priority(heur)
    count = g.color()
    return g, g.priorities(), g.colors(), count


@pytest.mark.parametrize("heur", HEURISTICS)
def test_golden_parity(gpu_ctx, golden, models, heur):
    for name in golden.graphs:
        N, V, E = golden.graph(name)
        g, p, c, count = gpu_run(gpu_ctx, N, V, E, heur, models)
        assert np.array_equal(p, golden.get(name, heur, "p")), (name, heur, "priorities")
        assert np.array_equal(c, golden.get(name, heur, "color")), (name, heur, "colors")
        assert count == (int(c.max()) if N else 1)
        assert count == O.validate(N, V, E, c)
        g.recolor(3)
        assert np.array_equal(g.colors(), golden.get(name, heur, "culb3")), (name, heur, "culberson")
        g.close()


def test_reference_models(gpu_ctx, golden, golden_ref):
    if not os.path.exists(os.path.join(R.MODELS, "m3.gnn")):
        pytest.skip("reference model files not present (oracle/_ref/models)")
    for L in (2, 3, 4):
        m = gcn.Model.load(gpu_ctx, os.path.join(R.MODELS, f"m{L}.gnn"))
        for name in ("er1500", "rmat11", "bridged"):
            N, V, E = golden.graph(name)
            g = gcn.Graph(gpu_ctx, N, V, E)
            g.priority("GNN", m)
            g.color()
            assert np.array_equal(g.priorities(), golden_ref[f"{name}/GNN{L}/p"]), (name, L)
            assert np.array_equal(g.colors(), golden_ref[f"{name}/GNN{L}/color"]), (name, L)


def test_rmat22_gnn3_reference_model_matches_the_reference(gpu_ctx):
    """The headline configuration at full size: R-MAT scale 22 (4.2 M vertices, 128 M directed
    edges, hubs of up to 162,886 neighbours -- the giant-hub path, the cluster core and both ticket
    streams all run), the reference's own models/m3.gnn.  Priorities (bit patterns) and colors
    must equal the reference's gnn_internal_par on the same graph, run here on the host cores."""
    if not (R.available() and R.has_models()):
        pytest.skip("the compiled reference and its model files are not present (oracle/_ref)")
    N, V, E = gcn.gen_rmat(1 << 22, 16, 2)
    m = gcn.Model.load(gpu_ctx, os.path.join(R.MODELS, "m3.gnn"))
    g = gcn.Graph(gpu_ctx, N, V, E)
    g.priority("GNN", m)
    count = g.color()
    p, c = g.priorities(), g.colors()
    g.close()
    m.close()
    R.set_threads(os.cpu_count() or 1)
    job = R.GnnJob(N, V, E, 3)
    c_ref = job.run()[:N].copy()
    p_ref = job.p[:N].copy()
    job.close()
    assert np.array_equal(p.view(np.uint64), p_ref.view(np.uint64)), "GNN3 priorities differ from the reference"
    assert np.array_equal(c, c_ref), "colors differ from the reference"
    assert count == int(c_ref.max())


def er65k():
    # the plain CPU-runnable configuration: ER n=65,536, 524,288 undirected edges, seed 1
    return gcn.gen_er(65536, 524288, 1)


@pytest.mark.parametrize("heur", HEURISTICS)
def test_er65k_all_heuristics(gpu_ctx, golden, models, heur):
    N, V, E = er65k()
    g, p, c, count = gpu_run(gpu_ctx, N, V, E, heur, models)
    if heur.startswith("GNN"):
        params, md = golden.model(int(heur[3:]))
        po = O.ordering("GNN", N, V, E, params, md)
    else:
        po = O.ordering(heur, N, V, E)
    assert np.array_equal(p, po), heur
    co, _ = O.greedy_color(N, V, E, po)
    assert np.array_equal(c, co), heur
    assert count == int(co.max())


@pytest.mark.parametrize("scale,heur", [(16, "GNN3"), (16, "SL"), (18, "GNN3"), (18, "LF"), (18, "SLL"),
                                        (18, "LLF"), (18, "FF")])
def test_rmat_vs_oracle(gpu_ctx, golden, models, scale, heur):
    N, V, E = gcn.gen_rmat(1 << scale, 16, 2)
    g, p, c, count = gpu_run(gpu_ctx, N, V, E, heur, models)
    if heur.startswith("GNN"):
        params, md = golden.model(int(heur[3:]))
        po = O.ordering("GNN", N, V, E, params, md)
    else:
        po = O.ordering(heur, N, V, E)
    assert np.array_equal(p, po)
    co, _ = O.greedy_color(N, V, E, po)
    assert np.array_equal(c, co)
    g.recolor(2)
    assert np.array_equal(g.colors(), O.culberson(N, V, E, co, 2))


def test_mesh_graphs_culberson(gpu_ctx, golden, models):
    """Mesh-like inputs with GNN4 + JP + 9 Culberson recolorings (the -c 10 protocol)."""
    for N, V, E in (gcn.gen_rgg2d(1 << 16, float(np.sqrt(12 / (np.pi * (1 << 16)))), 3),
                    gcn.gen_stencil27(24, 24, 24)):
        g, p, c, count = gpu_run(gpu_ctx, N, V, E, "GNN4", models)
        params, md = golden.model(4)
        po = O.ordering("GNN", N, V, E, params, md)
        assert np.array_equal(p, po)
        co, _ = O.greedy_color(N, V, E, po)
        assert np.array_equal(c, co)
        counts = [count]
        for _ in range(9):
            counts.append(g.recolor(1))
        assert all(b <= a for a, b in zip(counts, counts[1:]))
        assert np.array_equal(g.colors(), O.culberson(N, V, E, co, 9))


def _star(n):
    """Vertex 0 joined to all others: one hub of n - 1 neighbours whose layer-0 id features
    (v / n, dyadic for n a power of two) make exact rounding ties in its FP32 sum."""
    V = np.concatenate([[0, n - 1], np.arange(n, 2 * n - 1)]).astype(np.uint32)
    E = np.concatenate([np.arange(1, n), np.zeros(n - 1)]).astype(np.uint32)
    return n, V, E


def _one_graph_batch_priorities(ctx, graph, model, hub_degree):
    t = gcn.default_tuning()
    t.hub_degree = hub_degree
    t.warp_degree = min(t.warp_degree, hub_degree)
    b = gcn.Batch(ctx, graphs=[graph])
    b.tuning = t
    b.color("GNN", model)
    p, c = b.priorities(), b.colors()
    b.close()
    return p, c


@pytest.mark.parametrize("L", [2, 3, 4])
def test_hub_exact_sums_match_oracle(gpu_ctx, golden, models, L):
    """Hubs (more than the hub degree) have their FP32 neighbour chains evaluated exactly by whole
    warps, 1,024 values per step (binade increments, parity-resolved ties, serial adds where the
    sum changes binade).  Lowering the hub degree sends many vertices of small graphs there, the
    star's id features make exact ties; every priority must still equal the oracle's bit for bit."""
    params, md = golden.model(L)
    graphs = [gcn.gen_rmat(1 << 15, 16, 9), _star(1 << 17), _star(100000), gcn.gen_er(20000, 400000, 4)]
    for graph in graphs:
        N, V, E = graph
        p_ref = O.ordering("GNN", N, V, E, params, md)
        c_ref, _ = O.greedy_color(N, V, E, p_ref)
        for hub in (64, 1024):
            p, c = _one_graph_batch_priorities(gpu_ctx, graph, models[L], hub)
            assert np.array_equal(p, p_ref), (N, hub, "priorities")
            assert np.array_equal(c, c_ref), (N, hub, "colors")


@pytest.mark.parametrize("fuse", ["1", "0"])
def test_isolated_vertices_match_oracle(golden, fuse):
    """Vertices without neighbours run every layer at once (k_gnn_isolated, the FMA prefix over the
    inputs common to all of them evaluated once per CTA) unless GC_GNN_FUSE_ISOLATED=0; either way
    every priority equals the oracle's bit for bit, for 2, 3 and 4 layers, in a plain graph and in
    a batch (segment-local id features)."""
    ctx = _ctx_with({"GC_GNN_FUSE_ISOLATED": fuse})
    N0, V0, E0 = gcn.gen_rmat(1 << 16, 4, 11)  # R-MAT with a sparse edge factor: many isolated ids
    graphs = [(N0, V0, E0), (3000, np.zeros(3001, np.uint32), np.zeros(0, np.uint32))]
    for L in (2, 3, 4):
        params, md = golden.model(L)
        m = gcn.Model(ctx, params, md)
        for N, V, E in graphs:
            g = gcn.Graph(ctx, N, V, E)
            g.priority("GNN", m)
            assert np.array_equal(g.priorities(), O.ordering("GNN", N, V, E, params, md)), (fuse, L, N)
            g.close()
        b = gcn.Batch(ctx, graphs=graphs)
        b.color("GNN", m)
        p = b.priorities()
        off = 0
        for N, V, E in graphs:
            assert np.array_equal(p[off:off + N], O.ordering("GNN", N, V, E, params, md)), (fuse, L, "batch", N)
            off += N
        b.close()
        m.close()
    assert int(np.sum(np.diff(V0.astype(np.int64)) == 0)) > 1000
    ctx.close()


def _ctx_with(env: dict):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return gcn.Context(int(os.environ.get("GC_DEVICE", "0")))
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("core,light,block,decide", [("0", "0", "16", "1"), ("0", "2", "16", "1"), ("64", "2", "1", "1"),
                                                     ("5000", "6", "7", "1"), ("32768", "0", "16", "1"),
                                                     ("32768", "2", "16", "1"), ("4097", "2", "64", "1"),
                                                     ("32768", "2", "1", "1"), ("32768", "2", "16", "0"),
                                                     ("777", "2", "3", "0")])
def test_jp_core_sizes_give_the_oracle_colors(golden, core, light, block, decide):
    """The first GC_JP_CORE tickets are colored inside one thread-block cluster (colors exchanged
    through distributed shared memory; early decisions from published seen colors unless
    GC_JP_CORE_DECIDE=0), the rest by the ticket kernel, split into a heavy and a light stream when
    GC_JP_LIGHT_WARPS > 0, with GC_JP_CORE_BLOCK consecutive core tickets per CTA: any combination
    gives the greedy coloring of the priorities, for float (GNN) and integer (LF) keys and after
    Culberson rounds."""
    ctx = _ctx_with({"GC_JP_CORE": core, "GC_JP_LIGHT_WARPS": light, "GC_JP_CORE_BLOCK": block,
                     "GC_JP_CORE_DECIDE": decide})
    params, md = golden.model(3)
    m = gcn.Model(ctx, params, md)
    for N, V, E in (gcn.gen_rmat(1 << 17, 16, 2), gcn.gen_er(30000, 300000, 8)):
        g = gcn.Graph(ctx, N, V, E)
        for heur in ("GNN", "LF"):
            g.priority(heur, m if heur == "GNN" else None)
            g.color()
            p = g.priorities()
            c_ref, _ = O.greedy_color(N, V, E, p)
            assert np.array_equal(g.colors(), c_ref), (core, light, block, decide, N, heur)
        g.recolor(2)
        assert np.array_equal(g.colors(), O.culberson(N, V, E, c_ref, 2)), (core, light, block, decide, N)
        g.close()
    m.close()
    ctx.close()


def test_user_priorities(gpu_ctx):
    N, V, E = gcn.gen_rmat(1 << 12, 8, 21)
    rng = np.random.default_rng(0)
    for p in (rng.integers(0, 5, N).astype(np.float64),                 # many ties
              rng.normal(size=N),                                      # negatives, non-integers
              np.where(rng.random(N) < 0.5, -0.0, 0.0),                # -0.0 equals +0.0
              rng.integers(0, 2**32 - 1, N).astype(np.float64)):       # full uint32 range
        g = gcn.Graph(gpu_ctx, N, V, E)
        g.set_priority(p)
        g.color()
        co, _ = O.greedy_color(N, V, E, p)
        assert np.array_equal(g.colors(), co)
        assert np.array_equal(g.priorities(), p)
    g = gcn.Graph(gpu_ctx, N, V, E)
    bad = np.zeros(N)
    bad[5] = np.nan
    with pytest.raises(gcn.GCError) as e:
        g.set_priority(bad)
    assert e.value.name == "GC_ERR_INVALID"


def test_deterministic_repeats(gpu_ctx, models):
    N, V, E = gcn.gen_rmat(1 << 15, 16, 5)
    g = gcn.Graph(gpu_ctx, N, V, E)
    ref = None
    for _ in range(3):
        g.priority("GNN", models[3])
        g.color()
        c = g.colors()
        if ref is None:
            ref = c
        assert np.array_equal(c, ref)


def test_call_order_and_bad_input(gpu_ctx):
    N, V, E = gcn.gen_er(100, 300, 1)
    g = gcn.Graph(gpu_ctx, N, V, E)
    with pytest.raises(gcn.GCError) as e:
        g.color()
    assert e.value.name == "GC_ERR_STATE"
    with pytest.raises(gcn.GCError) as e:
        g.priority("GNN")  # no model
    assert e.value.name == "GC_ERR_INVALID"
    bad = E.copy()
    bad[3] = 1000  # out of range
    with pytest.raises(gcn.GCError) as e:
        gcn.Graph(gpu_ctx, N, V, bad)
    assert e.value.name == "GC_ERR_INVALID"
    # the context is still usable
    g.priority("LF")
    assert g.color() > 0


def test_bounded_wait_expires_cleanly(monkeypatch):
    """A context whose wait limit is 0 gives up on the first uncolored predecessor: the kernel
    raises its error flag and returns, the host reports GC_ERR_DEVICE, and the context stays usable."""
    monkeypatch.setenv("GC_SPIN_LIMIT", "0")
    ctx = gcn.Context(int(os.environ.get("GC_DEVICE", "0")))
    n = 200000
    I = np.arange(n - 1, dtype=np.uint32)
    N, V, E = gcn.csr_from_pairs(n, I, I + 1)  # a path: FF makes one chain of n waits
    g = gcn.Graph(ctx, N, V, E)
    g.priority("FF")
    with pytest.raises(gcn.GCError) as e:
        g.color()
    assert e.value.name == "GC_ERR_DEVICE"
    # no waits at all: succeeds on the same context
    N2, V2, E2 = gcn.csr_from_pairs(1000, np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    g2 = gcn.Graph(ctx, N2, V2, E2)
    g2.priority("LF")
    assert g2.color() == 1
    g.close()
    g2.close()
    ctx.close()


def test_legacy_abi(golden):
    """The reference-named entry points (include/coloring.h etc.) with host buffers."""
    L = gcn.legacy
    for name in ("er1500", "rmat11", "bridged", "path7"):
        N, V, E = golden.graph(name)
        for fn, h in (("first_fit_ordering", "FF"), ("largest_degree_first_ordering", "LF"),
                      ("largest_log_degree_first_ordering", "LLF"), ("smallest_degree_last_ordering", "SL"),
                      ("smallest_log_degree_last_ordering", "SLL")):
            p = L.ordering(fn, N, V, E)
            assert np.array_equal(p, golden.get(name, h, "p")), (name, fn)
            c = L.coloring("jones_plassmann_coloring", N, V, E, p)
            assert np.array_equal(c, golden.get(name, h, "color")), (name, fn)
            assert np.array_equal(L.coloring("greedy_coloring", N, V, E, p), c)
            assert L.validate(N, V, E, c) == int(c.max())
        for fn, h in (("first_fit_coloring", "FF"), ("largest_degree_first_coloring_par", "LF"),
                      ("largest_log_degree_first_coloring", "LLF"), ("smallest_degree_last_coloring_par", "SL"),
                      ("smallest_log_degree_last_coloring", "SLL")):
            assert np.array_equal(L.coloring(fn, N, V, E), golden.get(name, h, "color")), (name, fn)
        params, md = golden.model(3)
        p = L.graph_sage(params, md, N, V, E)
        assert np.array_equal(p, golden.get(name, "GNN3", "p"))
        bad = golden.get(name, "FF", "color").copy()
        if len(E):
            u = int(np.argmax(np.diff(V) > 0))
            bad[u] = bad[E[V[u]]]
            assert L.validate(N, V, E, bad) == 0


def test_legacy_gnn_ordering_reads_model_dir(golden, tmp_path, monkeypatch):
    for L in (2, 3, 4):
        params, md = golden.model(L)
        gcn.model_write(str(tmp_path / f"m{L}.gnn"), params, md)
    monkeypatch.setenv("GC_MODEL_DIR", str(tmp_path))
    N, V, E = golden.graph("rmat11")
    for L in (2, 3, 4):
        p = gcn.legacy.ordering("gnn_ordering", N, V, E, layers=L)
        assert np.array_equal(p, golden.get("rmat11", f"GNN{L}", "p"))


def test_cli_output_lines(golden, tmp_path):
    """./coloring prints the reference's line format with the oracle's color counts."""
    for L in (2, 3, 4):
        params, md = golden.model(L)
        gcn.model_write(str(tmp_path / f"m{L}.gnn"), params, md)
    N, V, E = golden.graph("er1500")
    path = str(tmp_path / "g.mtx")
    gcn.mtx_write(path, N, V, E)
    env = dict(os.environ, GC_MODEL_DIR=str(tmp_path))
    r = subprocess.run([os.path.join(PKG, "cli", "coloring"), "-g", path, "-c", "2", "1", "8"],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.rstrip("\n").split("\n")
    names = [ln.split()[0] for ln in lines]
    assert names == [f"{h}_{i}" for h in ("FF", "LF", "LLF", "SL", "SLL", "GNN2", "GNN3", "GNN4") for i in (0, 1)]
    for ln in lines:
        parts = ln.split(" ")
        assert parts[-1] == ""  # trailing space as in src/runner.c:166-168
        name, colors, times = parts[0], int(parts[1]), parts[2:-1]
        assert len(times) == 3 and all(len(t.split(".")[1]) == 6 for t in times)
        h, i = name.split("_")
        want = golden.get("er1500", h, "color")
        if i == "1":
            want = O.culberson(N, V, E, want, 1)
        assert colors == int(want.max()), name
    q = subprocess.run([os.path.join(PKG, "cli", "coloring"), "-g", path, "-q"], capture_output=True, text=True,
                       timeout=600, env=env)
    assert q.returncode == 0, q.stderr
    vals = [int(x) for x in q.stdout.split()]
    expect = [int(golden.get("er1500", h, "color").max()) for h in ("FF", "LF", "LLF", "SL", "SLL")]
    inc = np.load(os.path.join(GOLDEN, "golden_incidence.npz"))
    expect += [int(inc[f"er1500/{fn}/color"].max()) for fn in
               ("incidence_degree_ordering", "saturation_degree_ordering_alt", "saturation_degree_ordering")]
    expect += [int(golden.get("er1500", f"GNN{L}", "color").max()) for L in (2, 3, 4)]
    assert vals == expect
    qf = subprocess.run([os.path.join(PKG, "cli", "coloring"), "-g", path, "-q", "-f"], capture_output=True,
                        text=True, timeout=600, env=env)
    valsf = [int(x) for x in qf.stdout.split()]
    assert valsf[2] == valsf[4] == valsf[5] == valsf[6] == valsf[7] == 0  # -f skips LLF, SLL, ID, SDA, SD


def test_reference_main_prints_what_the_cli_prints(golden, tmp_path):
    """INTEGRATION.md option 2 on the GPU: the reference's own main.c linked against this library
    prints the same lines as cli/coloring (names, color counts, column count; times masked), in
    runner mode with Culberson and in quick mode."""
    ref_main = os.path.join(os.path.dirname(R.PATH), "coloring_main")
    if not os.path.exists(ref_main):
        pytest.skip("the reference's main.c was not compiled here (reference sources absent at build time)")
    for L in (2, 3, 4):
        gcn.model_write(str(tmp_path / f"m{L}.gnn"), *golden.model(L))
    N, V, E = golden.graph("er1500")
    path = str(tmp_path / "g.mtx")
    gcn.mtx_write(path, N, V, E)
    env = dict(os.environ, GC_MODEL_DIR=str(tmp_path))

    def run(exe, *args):
        r = subprocess.run([exe, "-g", path, *args], capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0, (exe, r.stderr)
        return r.stdout

    def masked(out):
        return [ln.split(" ")[:2] + [len(ln.split(" "))] for ln in out.rstrip("\n").split("\n")]

    cli = os.path.join(PKG, "cli", "coloring")
    a, b = run(ref_main, "-c", "3", "1", "4"), run(cli, "-c", "3", "1", "4")
    assert masked(a) == masked(b)
    assert len(masked(a)) == 8 * 3
    assert run(ref_main, "-q") == run(cli, "-q")
    assert run(ref_main, "-q", "-f") == run(cli, "-q", "-f")


def test_incidence_orderings_color_like_the_reference(gpu_ctx, golden):
    """JP on the ID / SDA / SD priorities (host orderings) gives the reference's colors."""
    inc = np.load(os.path.join(GOLDEN, "golden_incidence.npz"))
    for name in golden.graphs:
        N, V, E = golden.graph(name)
        for fn in ("incidence_degree_ordering", "saturation_degree_ordering_alt", "saturation_degree_ordering"):
            p = inc[f"{name}/{fn}/p"]
            g = gcn.Graph(gpu_ctx, N, V, E)
            g.set_priority(p)
            g.color()
            assert np.array_equal(g.colors(), inc[f"{name}/{fn}/color"]), (name, fn)
            g.close()


def test_recolor_from_caller_colors(gpu_ctx):
    """Culberson rounds on a coloring the caller uploaded (colors far above max degree + 1): the keys
    are the caller's colors, so the result is the greedy coloring in that order (oracle)."""
    N, V, E = gcn.gen_rmat(1 << 12, 8, 77)
    g = gcn.Graph(gpu_ctx, N, V, E)
    user = (np.arange(N, dtype=np.int32) * 7 + 3)  # all distinct, so proper; up to ~28,000
    g.set_colors(user)
    g.recolor(1)
    ref, _ = O.greedy_color(N, V, E, user.astype(np.float64))
    assert np.array_equal(g.colors(), ref)
    g.recolor(2)  # then rounds on the library's own colors
    ref2 = ref
    for _ in range(2):
        ref2, _ = O.greedy_color(N, V, E, ref2.astype(np.float64))
    assert np.array_equal(g.colors(), ref2)
    g.close()


@pytest.mark.parametrize("heur", ["LF", "GNN3"])
def test_culberson_classes_match_tickets(gpu_ctx, heur):
    """Class-by-class Culberson rounds give the same colors as the oracle's rounds, on skewed and
    mesh-like graphs."""
    params, md = gcn.synthetic_model(3, 1003)
    m = gcn.Model(gpu_ctx, params, md)
    for N, V, E in (gcn.gen_rmat(1 << 14, 16, 5), gcn.gen_stencil27(24, 24, 24)):
        g = gcn.Graph(gpu_ctx, N, V, E)
        g.priority("GNN" if heur == "GNN3" else heur, m if heur == "GNN3" else None)
        g.color(4)
        p = O.ordering("GNN" if heur == "GNN3" else heur, N, V, E, params, md)
        c, _ = O.greedy_color(N, V, E, p)
        for _ in range(4):
            c, _ = O.greedy_color(N, V, E, c.astype(np.float64))
        assert np.array_equal(g.colors(), c), (heur, N)
        g.close()
    m.close()
