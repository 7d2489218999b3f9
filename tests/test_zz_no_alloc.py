"""GPU test of gc_gnn_priority_noalloc, the entry point for callers that may not allocate device
memory (a serving loop with a fixed HBM budget, a host framework that owns all device memory, a
path that cannot afford cudaMalloc's implicit synchronisation).

It must give exactly the priorities of the regular entry point, gc_priority(GC_GNN) (tolerance 0,
as every GraphSAGE parity test here), on two calls in a row with different graphs and models --
the second call reuses the shared scratch array the first one left behind and, being the first to
run a hidden layer, must load no code and allocate nothing -- and it must refuse
graphs larger than its fixed scratch.  Inputs and outputs are device buffers the test allocates
itself, as such a caller would."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

import gnn_coloring as gcn

pytestmark = pytest.mark.gpu

MAX_V = 65536  # GC_NOALLOC_MAX_VERTICES in include/gnn_coloring.h
fn = gcn.lib.gc_gnn_priority_noalloc
fn.restype = C.c_int
fn.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]


def device():
    return torch.device("cuda", int(os.environ.get("GC_DEVICE", "0")))


def regular_priorities(ctx, N, V, E, params, md):
    model = gcn.Model(ctx, params, md)
    g = gcn.Graph(ctx, N, V, E)
    g.priority("GNN", model)
    p = g.priorities().astype(np.float32)  # exact: the doubles are widened floats
    g.close()
    model.close()
    return p


def noalloc_priorities(N, V, E, params, md):
    dev = device()
    dV = torch.from_numpy(np.ascontiguousarray(V).view(np.int32)).to(dev)
    dE = torch.from_numpy(np.ascontiguousarray(E).view(np.int32) if len(E) else np.zeros(1, np.int32)).to(dev)
    dP = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(dev)
    out = torch.full((max(N, 1),), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    free_before = torch.cuda.mem_get_info(dev)[0]
    status = fn(N, dV.data_ptr(), dE.data_ptr(), len(params), md, dP.data_ptr(), out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    free_after = torch.cuda.mem_get_info(dev)[0]
    return status, out[:N].cpu().numpy(), free_before - free_after


def test_noalloc_matches_regular_entry_point_twice(gpu_ctx):
    # The 2-layer model first: the second call is the first to run a hidden layer, so it would load
    # that kernel (and allocate for its code) if the first call had not loaded every kernel.
    cases = [
        (gcn.gen_er(20000, 100000, 3), gcn.synthetic_model(2, 1002)),   # no hidden layer
        (gcn.gen_rmat(1 << 15, 16, 7), gcn.synthetic_model(3, 1003)),   # hubs, isolated vertices, a hidden layer
    ]
    for call, ((N, V, E), (params, md)) in enumerate(cases):
        assert N <= MAX_V
        want = regular_priorities(gpu_ctx, N, V, E, params, md)
        status, got, grown = noalloc_priorities(N, V, E, params, md)
        assert status == 0, gcn.STATUS.get(status, status)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"call {call}: priorities differ"
        if call > 0:  # the scratch array was set up by the first call: nothing is allocated now
            assert grown == 0


def test_noalloc_rejects_graphs_beyond_its_scratch():
    dev = device()
    dummy = torch.zeros(16, dtype=torch.int32, device=dev)
    params, md = gcn.synthetic_model(2, 1)
    dP = torch.from_numpy(params).to(dev)
    out = torch.zeros(16, dtype=torch.float32, device=dev)
    status = fn(MAX_V + 1, dummy.data_ptr(), dummy.data_ptr(), len(params), md, dP.data_ptr(), out.data_ptr(), None)
    assert gcn.STATUS[status] == "GC_ERR_INVALID"
