"""Serving (gc_serve_*): continuous batching of arriving jobs over device-resident pools, admission
by HBM budget, per-job latency.  The property that matters: every job's colors and color count are
those of its graph colored alone -- by the plain device path and by the oracle -- whatever it was
batched with, whichever lane ran it and whatever else ran beside it.

GPU tests call the library's serving entry points through the C ABI (gnn_coloring.Server)."""
import threading

import numpy as np
import pytest

import gnn_coloring as gcn

MODEL_MD = 100


def _oracle():
    from oracle import restatement as orc
    return orc


def _small_graphs(k, seed0=500, n_min=60, n_max=4000):
    return [gcn.gen_mixed(seed0 + i, n_min, n_max)[:3] for i in range(k)]


def _heur_args(name):
    """(heuristic, layers) of a job from a reference-style name: FF, LF, LLF, SL, SLL, GNN2..GNN4."""
    if name.startswith("GNN"):
        return "GNN", int(name[3:])
    return name, 0


def _alone(ctx, models, graph, name, recolor=0):
    N, V, E = graph
    heur, layers = _heur_args(name)
    g = gcn.Graph(ctx, N, V, E)
    g.priority(heur, models[layers] if heur == "GNN" else None)
    count = g.color(recolor)
    col = g.colors()
    g.close()
    return col, count


def test_config_defaults():
    c = gcn.serve_config_default()
    assert c.lanes == 4 and c.hbm_budget == 0
    assert c.slot_graphs == 4096 and c.slot_vertices == 1 << 22 and c.slot_edges == 1 << 26
    assert c.batch_max_job_vertices == 1 << 17


# ---- device ------------------------------------------------------------------------------------

@pytest.fixture(scope="module")
def model_params():
    return {L: gcn.synthetic_model(L, 1000 + L, MODEL_MD) for L in (2, 3, 4)}


@pytest.fixture(scope="module")
def models(gpu_ctx, model_params):
    return {L: gcn.Model(gpu_ctx, *model_params[L]) for L in (2, 3, 4)}


def _server(model_params, **kw):
    kw.setdefault("slot_vertices", 1 << 18)
    kw.setdefault("slot_edges", 1 << 22)
    kw.setdefault("slot_graphs", 512)
    return gcn.Server(models=[model_params[L] for L in (2, 3, 4)], **kw)


@pytest.mark.gpu
def test_mixed_jobs_from_many_threads_equal_alone(gpu_ctx, models, model_params):
    """Small batched jobs, large jobs run alone, SL/SLL, Culberson rounds, all heuristics, submitted
    from four host threads at once: each result equals the same graph colored alone."""
    rng = np.random.default_rng(7)
    graphs = _small_graphs(40)
    graphs += [gcn.gen_rmat(1 << 13, 16, 31), gcn.gen_rmat(5000, 12, 32), gcn.gen_er(9000, 60000, 33)]
    names = ["FF", "LF", "LLF", "SL", "SLL", "GNN2", "GNN3", "GNN4"]
    jobs = []
    for i, gr in enumerate(graphs):
        for _ in range(2):
            jobs.append((gr, names[int(rng.integers(len(names)))], int(rng.choice([0, 0, 2]))))
    srv = _server(model_params, lanes=3, batch_max_job_vertices=4000)
    results = [None] * len(jobs)
    errors = []

    def worker(idx):
        try:
            ids = []
            for k in idx:
                gr, name, rc = jobs[k]
                heur, layers = _heur_args(name)
                ids.append((k, srv.submit(*gr, heuristic=heur, layers=layers, recolor=rc)))
            for k, jid in ids:
                results[k] = srv.wait(jid)
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(list(range(t, len(jobs), 4)),)) for t in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    orc = _oracle()
    for k, (gr, name, rc) in enumerate(jobs):
        col, info = results[k]
        ref_col, ref_count = _alone(gpu_ctx, models, gr, name, rc)
        assert np.array_equal(col, ref_col), (k, name, rc, "colors differ from the graph colored alone")
        assert info.colors == ref_count, (k, name, info.colors, ref_count)
        assert info.status == 0 and info.batch_jobs >= 1 and info.latency_ms >= info.run_ms >= 0
        if k < 12 and rc == 0 and not name.startswith("GNN"):
            N, V, E = gr
            p = orc.ordering(name, N, V, E)
            oc, _ = orc.greedy_color(N, V, E, p)
            assert np.array_equal(col, oc), (k, name, "colors differ from the oracle")
    assert st["p99_ms"] >= st["p50_ms"] > 0 and st["edges"] == sum(int(g[1][-1]) for g, _, _ in jobs)


@pytest.mark.gpu
def test_arrivals_join_the_next_batch(gpu_ctx, models, model_params):
    """One lane busy with a large job: small jobs that arrive meanwhile are admitted together as one
    batch when the lane frees up (continuous batching), and still equal their graphs alone."""
    srv = _server(model_params, lanes=1, batch_max_job_vertices=4000)
    big = gcn.gen_rmat(1 << 16, 16, 41)
    smalls = _small_graphs(30, seed0=900)
    jb = srv.submit(*big, heuristic="GNN", layers=3)
    ids = [srv.submit(*g, heuristic="LLF") for g in smalls]
    _, ib = srv.wait(jb)
    outs = [srv.wait(j) for j in ids]
    st = srv.stats()
    srv.close()
    assert ib.batch_jobs == 1
    sizes = [info.batch_jobs for _, info in outs]
    assert max(sizes) > 1, sizes  # arrivals during the large job were batched
    assert st["batched_jobs"] >= max(sizes)
    for g, (col, info) in zip(smalls, outs):
        ref_col, ref_count = _alone(gpu_ctx, models, g, "LLF")
        assert np.array_equal(col, ref_col) and info.colors == ref_count


@pytest.mark.gpu
def test_admission_by_hbm_budget(model_params):
    """Jobs that run alone are charged their device bytes: with room for one at a time they run one
    at a time (peak charge within the budget), and a job that can never fit is refused."""
    big = [gcn.gen_rmat(1 << 15, 16, 50 + i) for i in range(3)]
    charge = max(gcn.batch_device_bytes(1, g[0], int(g[1][-1]), "LF") for g in big)
    slot = gcn.batch_device_bytes(64, 1 << 14, 1 << 18, "GNN")
    budget = 2 * slot + charge + charge // 2
    srv = _server(model_params, lanes=2, hbm_budget=budget, slot_graphs=64, slot_vertices=1 << 14,
                  slot_edges=1 << 18, batch_max_job_vertices=2000)
    ids = [srv.submit(*g, heuristic="LF") for g in big]
    small = _small_graphs(5, seed0=3000, n_max=1500)
    sids = [srv.submit(*g, heuristic="FF") for g in small]
    infos = [srv.wait(j)[1] for j in ids]
    for j in sids:
        srv.wait(j)
    st = srv.stats()
    assert st["peak_reserved_bytes"] <= budget
    assert st["peak_reserved_bytes"] >= 2 * slot + min(gcn.batch_device_bytes(1, g[0], int(g[1][-1]), "LF")
                                                       for g in big)
    assert all(i.batch_jobs == 1 for i in infos)
    # a job larger than the whole budget is refused at submission; nothing of it is read but V[0], V[N]
    N = 1 << 24
    V = np.zeros(N + 1, np.uint32)
    V[-1] = 1 << 31
    E = np.zeros(4, np.uint32)
    with pytest.raises(gcn.GCError) as e:
        srv.submit(N, V, E, heuristic="LF")
    assert e.value.name == "GC_ERR_BUDGET"
    assert srv.stats()["rejected"] == 1
    srv.close()


@pytest.mark.gpu
def test_malformed_job_fails_alone(gpu_ctx, models, model_params):
    """A job whose CSR names a vertex outside its graph fails with GC_ERR_INVALID (the library's
    own range checks catch it before any kernel reads through it); its batch-mates still succeed."""
    srv = _server(model_params, lanes=1, batch_max_job_vertices=4000)
    blocker = gcn.gen_rmat(1 << 15, 16, 61)
    smalls = _small_graphs(6, seed0=4000, n_max=1500)
    N, V, E = smalls[3]
    E_bad = E.copy()
    E_bad[len(E_bad) // 2] = N + 5
    jobs = list(smalls)
    jobs[3] = (N, V, E_bad)
    jb = srv.submit(*blocker, heuristic="FF")
    ids = [srv.submit(*g, heuristic="FF") for g in jobs]
    srv.wait(jb)
    for k, jid in enumerate(ids):
        if k == 3:
            with pytest.raises(gcn.GCError) as e:
                srv.wait(jid)
            assert e.value.name == "GC_ERR_INVALID"
        else:
            col, info = srv.wait(jid)
            ref_col, ref_count = _alone(gpu_ctx, models, jobs[k], "FF")
            assert np.array_equal(col, ref_col) and info.colors == ref_count
    st = srv.stats()
    srv.close()
    assert st["failed"] == 1 and st["completed"] == len(jobs)


@pytest.mark.gpu
def test_open_loop_replay(gpu_ctx, models, model_params):
    """Poisson arrivals replayed by the library: every job completes, colors equal the graphs alone,
    and the latency percentiles are ordered."""
    rng = np.random.default_rng(11)
    pool = _small_graphs(12, seed0=7000, n_max=20000) + [gcn.gen_rmat(1 << 14, 16, 71)]
    J = 150
    which = [int(rng.integers(len(pool) - 1)) if rng.random() < 0.95 else len(pool) - 1 for _ in range(J)]
    names = [["FF", "LLF", "GNN3"][int(rng.integers(3))] for _ in range(J)]
    arrive = np.cumsum(rng.exponential(1.0 / 1500.0, J))
    srv = _server(model_params, lanes=4, batch_max_job_vertices=20000)
    heur = [_heur_args(n) for n in names]
    cols, infos = srv.replay(arrive, [pool[w] for w in which], [h for h, _ in heur], layers=[l for _, l in heur],
                             want_colors=True)
    st = srv.stats()
    srv.close()
    assert st["completed"] == J and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    cache = {}
    for i in range(J):
        key = (which[i], names[i])
        if key not in cache:
            cache[key] = _alone(gpu_ctx, models, pool[which[i]], names[i])
        assert np.array_equal(cols[i], cache[key][0]), (i, key)
        assert infos[i]["colors"] == cache[key][1]


@pytest.mark.gpu
def test_registered_graphs(gpu_ctx, models, model_params):
    """Device-resident graphs: jobs on them (batched or alone, concurrently with host-CSR jobs) equal
    their graphs colored alone; a graph with jobs outstanding cannot be released; releasing returns
    its budget charge."""
    srv = _server(model_params, lanes=3, batch_max_job_vertices=4000)
    base = srv.stats()["reserved_bytes"]
    graphs = _small_graphs(10, seed0=8000) + [gcn.gen_rmat(1 << 14, 16, 81)]
    ids = [srv.register(*g) for g in graphs]
    charged = sum(4 * (g[0] + 1) + 4 * int(g[1][-1]) for g in graphs)
    assert srv.stats()["reserved_bytes"] == base + charged
    names = ["FF", "LLF", "GNN3", "LF", "GNN2", "SLL"]
    jobs = []
    for rep in range(3):
        for k, gid in enumerate(ids):
            name = names[(k + rep) % len(names)]
            heur, layers = _heur_args(name)
            jobs.append((k, name, srv.submit_registered(gid, heur, layers)))
    host = [srv.submit(*graphs[k], heuristic="FF") for k in range(3)]
    with pytest.raises(gcn.GCError) as e:
        srv.unregister(ids[-1])
    assert e.value.name == "GC_ERR_STATE"
    for k, name, jid in jobs:
        col, info = srv.wait(jid)
        ref_col, ref_count = _alone(gpu_ctx, models, graphs[k], name)
        assert np.array_equal(col, ref_col), (k, name)
        assert info.colors == ref_count
    for k, jid in enumerate(host):
        col, _ = srv.wait(jid)
        assert np.array_equal(col, _alone(gpu_ctx, models, graphs[k], "FF")[0])
    st = srv.stats()
    assert st["batched_jobs"] > 0 and st["failed"] == 0
    for gid in ids:
        srv.unregister(gid)
    assert srv.stats()["reserved_bytes"] == base
    # a malformed CSR is refused at registration
    N, V, E = graphs[0]
    E_bad = E.copy()
    E_bad[0] = N
    with pytest.raises(gcn.GCError) as e:
        srv.register(N, V, E_bad)
    assert e.value.name == "GC_ERR_INVALID"
    srv.close()


@pytest.mark.gpu
def test_registered_replay(gpu_ctx, models, model_params):
    rng = np.random.default_rng(3)
    graphs = _small_graphs(8, seed0=9000, n_max=20000) + [gcn.gen_rmat(1 << 15, 16, 91)]
    srv = _server(model_params, lanes=4, batch_max_job_vertices=20000)
    ids = [srv.register(*g) for g in graphs]
    J = 120
    which = [int(rng.integers(len(graphs))) for _ in range(J)]
    names = [["FF", "LLF", "GNN3"][int(rng.integers(3))] for _ in range(J)]
    arrive = np.cumsum(rng.exponential(1.0 / 3000.0, J))
    heur = [_heur_args(n) for n in names]
    cols, infos = srv.replay_registered(arrive, [ids[w] for w in which], [h for h, _ in heur],
                                        layers=[l for _, l in heur], want_colors=True)
    st = srv.stats()
    srv.close()
    assert st["completed"] == J and st["failed"] == 0 and st["p99_ms"] >= st["p50_ms"] > 0
    cache = {}
    for i in range(J):
        key = (which[i], names[i])
        if key not in cache:
            cache[key] = _alone(gpu_ctx, models, graphs[which[i]], names[i])
        assert np.array_equal(cols[i], cache[key][0]) and infos[i]["colors"] == cache[key][1], (i, key)
