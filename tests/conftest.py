"""Shared test setup: import paths, the `gpu` marker, fixtures for golden data and graphs.

`-m "not gpu"` tests run anywhere (oracle vs golden vectors, host code, library exports);
`-m gpu` tests call the CUDA library through its C ABI and compare with the oracle."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gnn-coloring_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the library's C ABI")


class Golden:
    """Access to golden_synth.npz: graphs and the reference's outputs on them."""

    def __init__(self, path):
        self.z = np.load(path)
        self.graphs = sorted({k.split("/")[0] for k in self.z.files if not k.startswith("model/")})

    def graph(self, name):
        return int(self.z[f"{name}/N"]), self.z[f"{name}/V"], self.z[f"{name}/E"]

    def model(self, L):
        return self.z[f"model/GNN{L}/params"], int(self.z[f"model/GNN{L}/md"])

    def get(self, name, heur, what):
        return self.z[f"{name}/{heur}/{what}"]


@pytest.fixture(scope="session")
def golden():
    return Golden(os.path.join(GOLDEN, "golden_synth.npz"))


@pytest.fixture(scope="session")
def golden_ref():
    return np.load(os.path.join(GOLDEN, "golden_refmodels.npz"))


@pytest.fixture(scope="session")
def golden_mtx():
    return np.load(os.path.join(GOLDEN, "golden_mtx.npz"))


@pytest.fixture(scope="session")
def gpu_ctx():
    import gnn_coloring as gcn
    ctx = gcn.Context(int(os.environ.get("GC_DEVICE", "0")))
    yield ctx
    ctx.close()


HEURISTICS = ["FF", "LF", "LLF", "SL", "SLL", "GNN2", "GNN3", "GNN4"]
