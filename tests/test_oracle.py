"""The oracle (scalar C restatement of the reference) against the reference's golden vectors and,
where oracle/_ref/libref.so exists, against the reference's own compiled code on more graphs."""
import numpy as np
import pytest

from conftest import HEURISTICS
from oracle import reference as R
from oracle import restatement as O


def oracle_priorities(golden, name, heur):
    N, V, E = golden.graph(name)
    if heur.startswith("GNN"):
        params, md = golden.model(int(heur[3:]))
        return O.ordering("GNN", N, V, E, params, md)
    return O.ordering(heur, N, V, E)


@pytest.mark.parametrize("heur", HEURISTICS)
def test_oracle_matches_golden(golden, heur):
    for name in golden.graphs:
        N, V, E = golden.graph(name)
        p = oracle_priorities(golden, name, heur)
        assert np.array_equal(p, golden.get(name, heur, "p")), (name, heur, "priorities")
        color, _ = O.greedy_color(N, V, E, p)
        assert np.array_equal(color, golden.get(name, heur, "color")), (name, heur, "colors")
        assert O.validate(N, V, E, color) == (color.max() if N else 1)
        culb = O.culberson(N, V, E, color, 3)
        assert np.array_equal(culb, golden.get(name, heur, "culb3")), (name, heur, "culberson")


def test_culberson_never_increases_colors(golden):
    for name in golden.graphs:
        N, V, E = golden.graph(name)
        if not N:
            continue
        c = golden.get(name, "GNN3", "color")
        prev = c.max()
        for _ in range(4):
            c = O.culberson(N, V, E, c, 1)
            assert c.max() <= prev
            prev = c.max()


def test_oracle_reference_models(golden, golden_ref):
    """GNN priorities with the reference's trained models (weights not committed)."""
    import os
    import gnn_coloring as gcn
    if not os.path.exists(os.path.join(R.MODELS, "m3.gnn")):
        pytest.skip("reference model files not present (oracle/_ref/models)")
    for name in ("er1500", "rmat11", "bridged"):
        N, V, E = golden.graph(name)
        for L in (2, 3, 4):
            params, md = gcn.model_read(os.path.join(R.MODELS, f"m{L}.gnn"))
            p = O.ordering("GNN", N, V, E, params, md)
            assert np.array_equal(p, golden_ref[f"{name}/GNN{L}/p"])
            c, _ = O.greedy_color(N, V, E, p)
            assert np.array_equal(c, golden_ref[f"{name}/GNN{L}/color"])


@pytest.mark.skipif(not R.available(), reason="oracle/_ref/libref.so not built (reference tree absent)")
@pytest.mark.parametrize("graph", ["er", "rmat", "rgg"])
def test_oracle_vs_live_reference(graph):
    import gnn_coloring as gcn
    if graph == "er":
        N, V, E = gcn.gen_er(20000, 160000, 11)
    elif graph == "rmat":
        N, V, E = gcn.gen_rmat(1 << 14, 16, 12)
    else:
        N, V, E = gcn.gen_rgg2d(30000, float(np.sqrt(12 / (np.pi * 30000))), 13)
    R.set_threads(4)
    for h in ("FF", "LF", "LLF", "SL", "SLL"):
        p = O.ordering(h, N, V, E)
        assert np.array_equal(p, R.ordering(h, N, V, E)), h
        c, _ = O.greedy_color(N, V, E, p)
        assert np.array_equal(c, R.jp_color(N, V, E, p)), h
    for L in (2, 3, 4):
        params, md = gcn.synthetic_model(L, 77 + L)
        p = O.ordering("GNN", N, V, E, params, md)
        assert np.array_equal(p, R.graph_sage(params, md, N, V, E)), L
        c, _ = O.greedy_color(N, V, E, p)
        assert np.array_equal(c, R.jp_color(N, V, E, p)), L


def test_fp64_error_is_small(golden):
    """FP32 GNN priorities against an FP64 recomputation of the same model: the largest relative
    error stays below 1e-5, the tolerance the GPU priorities are held to."""
    N, V, E = golden.graph("er1500")
    for L in (2, 3, 4):
        params, md = golden.model(L)
        p32 = O.ordering("GNN", N, V, E, params, md)
        p64 = O.ordering("GNN64", N, V, E, params, md)
        rel = np.abs(p32 - p64).max() / max(np.abs(p64).max(), 1e-30)
        assert rel < 1e-5, (L, rel)
