#!/usr/bin/env python
"""Benchmark: GraphSAGE GNN3 priorities + Jones-Plassmann coloring on one B200 (plain path).

Workload (one "step" = one coloring job): R-MAT scale 22 (4,194,304 vertices), edge factor 16,
a/b/c/d = 0.57/0.19/0.19/0.05, seed 2, symmetrised, deduplicated, loops removed; GNN3 priorities
with the reference's own trained weights (models/m3.gnn, copied beside the compiled reference by
oracle/Makefile; seeded synthetic weights of the same layout only where that file is absent), then
JP.  Metric: colored edges/s = |E| (directed CSR length, the reference's |E|) / job time.

  value   device-resident: CSR on the GPU, CUDA events on the library's stream around K steps
          of gc_priority(GNN3) + gc_color; E (513 MB) is larger than L2, so no flush is needed.
          Per-graph preparation (once per upload) is reported beside it as prep_ms.
  e2e     the reference-facing call with host buffers: gnn_internal_par(N, V, E, ad, jp, p, color)
          from pinned memory, H2D of V/E and D2H of p/colors inside every timed step.
  roofline  the dominant bandwidth-bound kernel's algorithmic bytes per launch / its average
          event-timed duration, against MEASURED_PEAKS.json's HBM copy bandwidth.  Kernels with no
          byte roofline (the JP core, a chain of dependent colors; the exact hub sums, bound by
          their add arithmetic) are listed in `other_bounds` with their share of the job.
  cpu_baseline  the reference's own OpenMP code (oracle/_ref) on the host cores, same job; its
          p and colors are the parity check of the GPU result (`parity`), and the other
          workloads (`configs`) are checked the same way, Culberson round by round.

--impl reference runs the reference's own CPU implementation of the same job (rank 0 only), in a
process that never loads libgnncolor.so.
--gpus N > 1 runs N independent replicas, one per GPU (the path does not shard): weak scaling.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gnn-coloring_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "GNN3+JP colored edges/s"
UNIT = "edges/s"
MODEL_SEED = 1003  # synthetic GNN3 weights (seed 1000 + layers), only where the reference's model files are absent
REF_MODELS = os.path.join(ROOT, "oracle", "_ref", "models")
GRAPHS = {
    "rmat22": ("R-MAT scale 22, ef 16, a/b/c=0.57/0.19/0.19, seed 2", 22),
    "rmat18": ("R-MAT scale 18, ef 16, a/b/c=0.57/0.19/0.19, seed 2", 18),
    "er65k": ("Erdos-Renyi n=65536, m=524288, seed 1", None),
}


def model_file(layers: int):
    """The reference's own trained weights, models/m{L}.gnn (copied beside the compiled reference by
    oracle/Makefile), or None where they are absent."""
    path = os.path.join(REF_MODELS, f"m{layers}.gnn")
    return path if os.path.exists(path) else None


def model_desc(layers: int) -> str:
    if model_file(layers):
        return f"models/m{layers}.gnn (the reference's GNN{layers} weights)"
    return f"synthetic GraphSAGE-16 weights ({layers} layers, seed {1000 + layers}, md 100)"


def bench_config(workload_name: str, N: int, M: int) -> dict:
    """The `config` dict, identical in both arms."""
    return {"workload": f"{workload_name}_gnn3_jp", "graph": GRAPHS[workload_name][0], "N": N, "M": M,
            "heuristic": "GNN3", "model": model_desc(3),
            "l2": "inputs larger than L2 (E is %.0f MB); no flush" % (4 * M / 1e6)}


def workload(name: str):
    import gnn_coloring as gcn
    desc, scale = GRAPHS[name]
    if scale is not None:
        N, V, E = gcn.gen_rmat(1 << scale, 16, 2)
    else:
        N, V, E = gcn.gen_er(65536, 524288, 1)
    return desc, N, V, E


def workload_reference(name: str):
    """The same graph without loading the library: the library's R-MAT samples restated in numpy
    (synthgen), turned into a CSR by the reference's own mtx_to_graph_par, graph_sort_edges_par and
    graph_make_simple."""
    import synthgen
    from oracle import reference as R
    desc, scale = GRAPHS[name]
    I, J = synthgen.rmat_samples(1 << scale, 16, 2)
    V, E = R.csr_from_samples(1 << scale, I, J)
    return desc, 1 << scale, V, E


def cpu_info() -> dict:
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        nproc = len(os.sched_getaffinity(0))
    except AttributeError:
        nproc = os.cpu_count() or 1
    return {"cpu_model": model, "nproc": nproc}


def source_hash() -> str:
    """SHA-256 over the library's kernel and host sources and build flags: the ncu traffic figures
    are used only when they were captured on a build of these exact sources."""
    import hashlib
    h = hashlib.sha256()
    files = []
    for d in (os.path.join(PKG, "csrc"), os.path.join(ROOT, "include")):
        files += [os.path.join(d, f) for f in os.listdir(d)]
    files.append(os.path.join(PKG, "Makefile"))
    for path in sorted(files, key=lambda x: os.path.relpath(x, ROOT)):
        h.update(os.path.relpath(path, ROOT).encode())
        with open(path, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


# Algorithmic (compulsory) HBM bytes per launch of each kernel group, M = directed edges,
# N = vertices, P = predecessor entries (sum of predecessor counts).
def algorithmic_bytes(kernel: str, N: int, M: int, P: int) -> float:
    table = {
        "gnn_input": 4 * M + 4 * N + 8 * N + 64 * N,     # E, V, own layer-0 inputs, y rows
        "gnn_hidden": 4 * M + 4 * N + 64 * N + 64 * N,   # E, V, own x row, y row
        "gnn_output": 4 * M + 4 * N + 64 * N + 4 * N,    # E, V, own x row, key
        "gnn_table0": 4 * N + 8 * N,
        "jp_split": 4 * M + 4 * N + 4 * N + 4 * P + 4 * N + 4 * N,  # E, V, key, P written, pc, color reset
        "jp_color": 4 * N + 4 * N + 4 * N + 4 * P + 4 * N,          # order, V, pc, P read, color written
        "sort_pass": 4 * N * 4,                                      # keys+ids read and written
    }
    return float(table.get(kernel, 0))


def step_bytes(N: int, M: int, layers: int = 3) -> float:
    """Whole-job algorithmic bytes: GNN with L layers 4LM + (132L-124)N, JP 8M + 32N."""
    return 4 * layers * M + (132 * layers - 124) * N + 8 * M + 32 * N


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [ln.strip().split(", ") for ln in self.out.read().splitlines() if ln.strip()]
        self.out.close()
        os.unlink(self.out.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus: int, backend: str = "nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*).  The ranks are
    independent replicas: the process group carries only the barriers around the timed region and
    the max over ranks.  `backend` "gloo" runs the same steps on the CPU (tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The slowest rank's value (timing is reported as the max over ranks)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- the reference's CPU implementation -------------------------------------------------------

def run_reference(args):
    """The reference's own gnn_internal_par (src/gnn.c:78-83) with its own models/m3.gnn, on all
    host cores.  This process never loads libgnncolor.so: the graph comes from synthgen and the
    reference's CSR construction."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import reference as R
    if not (R.available() and R.has_models()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref.so and the reference's models were "
                                                              "not built (reference sources absent where build() ran)"}))
        return
    if GRAPHS[args.workload][1] is None:
        print(json.dumps({"impl": "reference", "unavailable": f"--impl reference generates R-MAT workloads only "
                                                              f"(asked: {args.workload})"}))
        return
    t0 = time.perf_counter()
    desc, N, V, E = workload_reference(args.workload)
    gen_s = time.perf_counter() - t0
    M = int(V[N])
    info = cpu_info()
    cores = info["nproc"]
    R.set_threads(cores)
    job = R.GnnJob(N, V, E, 3)
    for _ in range(args.warmup):
        job.run()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        job.run()
        times.append(time.perf_counter() - t0)
    colors = int(job.color[:N].max()) if N else 0
    job.close()
    total = sum(times)
    value = M * len(times) / total
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": bench_config(args.workload, N, M), "colors": colors, "graph_generation_s": gen_s,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", **info,
                         "sample": f"{args.steps} full GNN3+JP jobs through the reference's gnn_internal_par "
                                   f"(src/gnn.c:78-83) with its models/m3.gnn, OpenMP over {cores} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_baseline(N, V, E, budget_s: float = 20.0):
    """The reference's gnn_internal_par on the same graph, timed on all host cores; also returns its
    last p and colors, which the GPU result is checked against."""
    from oracle import reference as R
    info = cpu_info()
    cores = info["nproc"]
    if not (R.available() and R.has_models()):
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference", **info,
                "sample": "unavailable: oracle/_ref was not built"}, None, None
    R.set_threads(cores)
    job = R.GnnJob(N, V, E, 3)
    job.run()  # warm-up
    times = []
    t_start = time.perf_counter()
    while len(times) < 3 and time.perf_counter() - t_start < budget_s:
        t0 = time.perf_counter()
        job.run()
        times.append(time.perf_counter() - t0)
    p, c = job.p[:N].copy(), job.color[:N].copy()
    job.close()
    return ({"value": int(V[N]) * len(times) / sum(times), "unit": UNIT, "cores": cores, "kind": "reference", **info,
             "sample": f"{len(times)} full GNN3+JP jobs on the same graph (reference gnn_internal_par with its "
                       f"models/m3.gnn, {cores} OpenMP threads), best-effort within {budget_s:.0f} s"}, p, c)


def parity_entry(p_gpu, c_gpu, p_ref, c_ref, what: str) -> dict:
    if p_ref is None:
        return {"checked": False, "why": "reference not built"}
    return {"checked": True, "against": what,
            "p_bits_equal": bool(np.array_equal(np.asarray(p_gpu, np.float64).view(np.uint64),
                                                np.asarray(p_ref, np.float64).view(np.uint64))),
            "colors_equal": bool(np.array_equal(c_gpu, c_ref)), "colors": int(c_gpu.max()) if len(c_gpu) else 0,
            "colors_reference": int(c_ref.max()) if len(c_ref) else 0}


def prep_time_ms(ctx, N, V, E, reps: int = 5):
    """Per-graph preparation (CSR check, degree classes, hub lists, degree-sorted schedule, split
    tasks, the graph's device buffers) of a device-resident CSR: gc_graph_wrap_device on a device
    copy of V and E, which runs exactly that preparation.  One untimed call first, then the median
    and the minimum wall time of `reps` calls; not part of `value`."""
    import torch
    import gnn_coloring as gcn
    dV = torch.from_numpy(np.ascontiguousarray(V).view(np.int32)).cuda()
    dE = torch.from_numpy(np.ascontiguousarray(E).view(np.int32)).cuda()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps + 1):
        h = C.c_void_p()
        t0 = time.perf_counter()
        ctx.check(gcn.lib.gc_graph_wrap_device(ctx.h, N, int(V[N]), dV.data_ptr(), dE.data_ptr(), C.byref(h)),
                  "wrap device graph")
        ctx.sync()
        ts.append(1e3 * (time.perf_counter() - t0))
        gcn.lib.gc_graph_free(h)
    del dV, dE
    ts = ts[1:]
    return float(statistics.median(ts)), float(min(ts))


def rows_time_ms(ctx, model, N, V, E):
    """The GNN's feature-row order (k_gnn_rows, k_gnn_row_ids), built by the first GNN call after an
    upload: timed with the library's event pairs on a second graph, after one call has loaded the
    kernels and allocated the buffers and a re-upload of the same CSR has dropped the order.  Once
    per upload; not part of `value`."""
    import gnn_coloring as gcn
    g2 = gcn.Graph(ctx, N, V, E)
    g2.priority("GNN", model)  # allocates the graph's GNN buffers
    # the same CSR again: its preparation drops the row order, the buffers stay
    Vc, Ec = np.ascontiguousarray(V, np.uint32), np.ascontiguousarray(E, np.uint32)
    ctx.check(gcn.lib.gc_graph_reupload(ctx.h, g2.h, N, Vc.ctypes.data_as(C.POINTER(C.c_uint32)),
                                        Ec.ctypes.data_as(C.POINTER(C.c_uint32))), "re-upload")
    gcn.lib.gc_prof_enable(ctx.h, 1)
    g2.priority("GNN", model)
    ms = prof_totals(gcn, ctx).get("gnn_rows", {}).get("ms_per_step")
    gcn.lib.gc_prof_enable(ctx.h, 0)
    g2.close()
    return ms


def prof_totals(gcn, ctx, steps: int = 1):
    """The library's per-kernel event timings since gc_prof_enable, per step."""
    names = (C.c_char_p * 64)()
    tot = (C.c_double * 64)()
    cnt = (C.c_uint64 * 64)()
    gcn.lib.gc_prof_read.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    nk = gcn.lib.gc_prof_read(ctx.h, names, tot, cnt, 64)
    return {names[i].decode(): {"ms_per_step": tot[i] / steps, "launches_per_step": cnt[i] / steps}
            for i in range(min(nk, 64))}


def ncu_traffic(workload_name: str, kernel: str):
    """DRAM bytes per launch of `kernel` from profiles/ncu_traffic.json, when that file was captured
    on a build of the current sources; None otherwise."""
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(tpath) as f:
            d = json.load(f)
    except Exception:
        return None, "no capture"
    if d.get("source_sha256") != source_hash():
        return None, "capture is of other sources"
    v = d.get(workload_name, {}).get(kernel)
    return (v["dram_bytes_per_launch"] if isinstance(v, dict) else v), "ncu capture of this build"


# ---- our arm -------------------------------------------------------------------------------------

def run_ours(args):
    import torch
    import gnn_coloring as gcn
    world, rank, local = dist_setup(args.gpus)
    device = local
    torch.cuda.set_device(device)
    desc, N, V, E = workload(args.workload)
    M = int(V[N])

    ctx = gcn.Context(device)
    model = _model(ctx, gcn, 3)
    g = gcn.Graph(ctx, N, V, E)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", device))

    def step():
        g.priority("GNN", model)
        g.color(count=False)

    for _ in range(max(3, args.warmup)):
        step()
    colors_used = g.validate()
    assert colors_used > 0, "invalid coloring"
    p_gpu, c_gpu = g.priorities(), g.colors()

    sampler = ClockSampler(device)
    sampler.start()
    time.sleep(0.25)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launches
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    launches = ctx.launches - launches0
    elapsed_ms = e0.elapsed_time(e1)
    time.sleep(0.15)
    clocks = sampler.stop()
    elapsed_ms = max_over_ranks(elapsed_ms, world, torch.device("cuda", device))
    ms_per_step = elapsed_ms / args.steps
    value = world * M * args.steps / (elapsed_ms / 1e3)
    same_after = bool(np.array_equal(g.colors(), c_gpu))

    # per-kernel durations: event pairs on each kernel's own stream over a few more steps
    gcn.lib.gc_prof_enable(ctx.h, 1)
    prof_steps = max(1, min(args.steps, 5))
    for _ in range(prof_steps):
        step()
    kernels = prof_totals(gcn, ctx, prof_steps)
    gcn.lib.gc_prof_enable(ctx.h, 0)
    P = M // 2  # each undirected edge has exactly one predecessor end
    hbm_peak, peak_kind = peaks()
    byte_bound = [k for k in kernels if algorithmic_bytes(k, N, M, P) > 0]
    dominant = max(byte_bound, key=lambda k: kernels[k]["ms_per_step"]) if byte_bound else None
    other_bounds = {k: {"ms_per_step": v["ms_per_step"], "share": v["ms_per_step"] / ms_per_step,
                        "bound": "dependency chain (latency)" if k.startswith("jp_core") else
                        "FP32 add arithmetic (exact sums); the span from the layer's start on a high-priority "
                        "side stream, whose CTAs take SMs as the layer kernel's leave them, so it overlaps the "
                        "layer kernels' time" if k.startswith("gnn_hub") else "launch/latency"}
                    for k, v in kernels.items() if k not in byte_bound and v["ms_per_step"] > 0.05 * ms_per_step}
    roofline = None
    if dominant:
        per_launch_ms = kernels[dominant]["ms_per_step"] / max(kernels[dominant]["launches_per_step"], 1)
        alg = algorithmic_bytes(dominant, N, M, P)
        achieved = alg / (per_launch_ms / 1e3) / 1e9
        traffic, traffic_src = ncu_traffic(args.workload, dominant)
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": achieved / hbm_peak, "peak_kind": f"{peak_kind} (copy bandwidth)",
                    "algorithmic_bytes_per_launch": alg, "ms_per_launch": per_launch_ms, "traffic": traffic,
                    "traffic_source": traffic_src}
        if dominant.startswith("gnn_") and os.environ.get("GC_GNN_HUB_SIDE", "1") != "0":
            roofline["note"] = "timed live with the hub kernel running beside it on a second stream"
    job_bytes = step_bytes(N, M)
    step_roof = {"algorithmic_bytes": job_bytes, "achieved_gbs": job_bytes / (ms_per_step / 1e3) / 1e9,
                 "frac": job_bytes / (ms_per_step / 1e3) / 1e9 / hbm_peak}
    prep_ms, prep_min_ms = prep_time_ms(ctx, N, V, E) if world == 1 else (None, None)
    rows_ms = rows_time_ms(ctx, model, N, V, E) if world == 1 else None

    # e2e through the reference-facing entry point with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, N, V, E, torch)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic", "config": bench_config(args.workload, N, M),
        "parallelism": "replicas" if world > 1 else "single GPU", "colors": colors_used,
        "prep_ms": prep_ms, "prep_min_ms": prep_min_ms, "gnn_rows_ms": rows_ms,
        "prep_note": "per-graph preparation of a resident CSR (degree classes, hub lists, degree order, split "
                     "tasks: prep_ms; the GNN's feature-row order, built by the first GNN call after an upload: "
                     "gnn_rows_ms); once per upload, outside `value`, inside `e2e`",
        "gpu_launches": launches, "clocks": clocks, "roofline": roofline, "other_bounds": other_bounds, "step_roofline": step_roof,
        "kernels": kernels, "e2e": e2e,
    }
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, p_ref, c_ref = cpu_baseline(N, V, E)
        result["cpu_baseline"] = base
        parity = parity_entry(p_gpu, c_gpu, p_ref, c_ref, "reference gnn_internal_par (oracle/_ref), same graph "
                                                           "and model")
        parity["colors_same_after_timed_steps"] = same_after
        result["parity"] = parity
    if world == 1 and not args.no_configs:
        result["configs"] = run_configs(args, device)
    if world == 1 and not args.no_batch:
        result["batched"] = run_batched(args, device)
    if world == 1 and not args.no_serve:
        result["serving"] = run_serving(args, device)
    result["summary"] = summary_of(result)
    if rank == 0:
        print(json.dumps(result))
        print(json.dumps(result["summary"]), file=sys.stderr)
    g.close()
    model.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    bad = [k for k, v in parity_flags(result) if not v]
    if bad:
        raise SystemExit(f"parity failed: {bad}")


def parity_flags(result):
    """(name, ok) for every parity check the run made."""
    out = []
    par = result.get("parity")
    if par and par.get("checked"):
        out.append(("headline", par["p_bits_equal"] and par["colors_equal"] and par["colors_same_after_timed_steps"]))
    for name, cfg in (result.get("configs") or {}).items():
        par = cfg.get("parity") if isinstance(cfg, dict) else None
        if par and par.get("checked"):
            out.append((name, bool(par.get("all_equal"))))
    for name, r in ((result.get("batched") or {}).get("heuristics") or {}).items():
        out.append((f"batched_{name}", bool(r.get("colors_identical"))))
    srv = result.get("serving")
    if srv:
        out.append(("serving", bool(srv.get("color_counts_identical_to_alone"))))
    return out


def summary_of(result) -> dict:
    """A short digest placed last in the JSON line (and on stderr), so that a truncated tail of the
    output still shows the headline, e2e, the batched and served speed-ups and the parity checks."""
    s = {"value": result["value"], "ms_per_step": result["ms_per_step"],
         "e2e": (result.get("e2e") or {}).get("value"), "prep_ms": result.get("prep_ms"),
         "roofline_frac": (result.get("roofline") or {}).get("frac"),
         "step_roofline_frac": result["step_roofline"]["frac"],
         "cpu_baseline": (result.get("cpu_baseline") or {}).get("value")}
    b = result.get("batched")
    if b:
        s["batched"] = {k: {"speedup": round(v.get("speedup", 0), 2), "colors_identical": v.get("colors_identical")}
                        for k, v in b["heuristics"].items()}
    srv = result.get("serving")
    if srv:
        s["served"] = {f: {"speedup_edges_per_s": round(srv[f]["speedup_edges_per_s"], 2),
                           "speedup_jobs_per_s": round(srv[f]["speedup_jobs_per_s"], 2)}
                       for f in ("host_csr", "resident_csr") if f in srv}
    s["parity"] = {k: v for k, v in parity_flags(result)}
    return s


# ---- the other configurations: ER 65k with every heuristic, mesh-like graphs with Culberson ------

def _timed_jobs(ctx, g, heur, model, recolor, reps, torch, device):
    """Device time per job (priority + JP + recolor Culberson rounds) with CUDA events on the
    library's stream, after one warm-up job; returns (ms, colors)."""
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", device))
    g.priority(heur, model)
    colors = g.color(recolor)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        g.priority(heur, model)
        g.color(recolor, count=False)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, colors


def _model(ctx, gcn, L: int):
    """The GNN{L} model: the reference's own file where present, else seeded synthetic weights."""
    path = model_file(L)
    return gcn.Model.load(ctx, path) if path else gcn.Model(ctx, *gcn.synthetic_model(L, 1000 + L))


def _models(ctx, gcn):
    return {L: _model(ctx, gcn, L) for L in (2, 3, 4)}


def _reference_result(name, N, V, E):
    """The reference's p and colors for one heuristic (None where the reference was not built)."""
    from oracle import reference as R
    if not (R.available() and R.has_models()):
        return None, None
    R.set_threads(cpu_info()["nproc"])
    if name.startswith("GNN"):
        job = R.GnnJob(N, V, E, int(name[3:]))
        c = job.run()[:N].copy()
        p = job.p[:N].copy()
        job.close()
        return p, c
    if name in ("SL", "SLL"):
        return R.peel_par(name, N, V, E)
    p = R.ordering(name, N, V, E)
    return p, R.jp_color(N, V, E, p)


def run_configs(args, device):
    """The other workloads on the device-resident path, each checked against the reference's own
    code on the same graph and weights: Erdos-Renyi n = 65,536 with every heuristic, and the mesh
    graphs with GNN4 + JP + 9 Culberson rounds (the reference's -c 10), compared round by round."""
    import math
    import torch
    import gnn_coloring as gcn
    from oracle import reference as R
    ctx = gcn.Context(device)
    models = _models(ctx, gcn)
    out = {}
    # Erdos-Renyi n = 65,536, m = 524,288, seed 1: every heuristic, one coloring
    N, V, E = gcn.gen_er(65536, 524288, 1)
    g = gcn.Graph(ctx, N, V, E)
    rows, all_eq = {}, True
    for name in ("FF", "LF", "LLF", "SL", "SLL", "GNN2", "GNN3", "GNN4"):
        heur, m = ("GNN", models[int(name[3])]) if name.startswith("GNN") else (name, None)
        ms, colors = _timed_jobs(ctx, g, heur, m, 0, 10, torch, device)
        g.priority(heur, m)
        g.color()
        p_ref, c_ref = _reference_result(name, N, V, E)
        par = parity_entry(g.priorities(), g.colors(), p_ref, c_ref, "reference (oracle/_ref)")
        all_eq = all_eq and (not par["checked"] or (par["p_bits_equal"] and par["colors_equal"]))
        rows[name] = {"ms": ms, "colors": colors, "edges_per_s": len(E) / (ms / 1e3), "parity": par}
    g.close()
    out["er65k_all_heuristics"] = {"graph": "Erdos-Renyi n=65536, m=524288, seed 1", "N": N, "M": len(E),
                                   "models": {L: model_desc(L) for L in (2, 3, 4)}, "heuristics": rows,
                                   "parity": {"checked": R.available() and R.has_models(), "all_equal": all_eq}}
    # mesh-like graphs, GNN4 priorities + JP + 9 Culberson rounds (the reference's -c 10)
    n = 1 << 23
    for key, desc, gen in (
            ("rgg2d_8m_gnn4_c10", "2D random geometric graph, n=2^23, radius for mean degree 12, seed 1",
             lambda: gcn.gen_rgg2d(n, math.sqrt(12.0 / (math.pi * n)), 1)),
            ("stencil27_256_gnn4_c10", "3D 27-point stencil, 256^3 vertices", lambda: gcn.gen_stencil27(256, 256, 256))):
        N, V, E = gen()
        g = gcn.Graph(ctx, N, V, E)
        ms, colors = _timed_jobs(ctx, g, "GNN", models[4], 9, 3, torch, device)
        g.priority("GNN", models[4])
        first = g.color(0)
        p_gpu = g.priorities()
        rounds = [g.colors()]
        for _ in range(9):
            g.recolor(1)
            rounds.append(g.colors())
        g.close()
        entry = {"graph": desc, "N": N, "M": len(E), "model": model_desc(4), "ms_per_job": ms,
                 "edges_per_s": len(E) / (ms / 1e3), "colors_first": first, "colors_after_9_culberson": colors}
        if R.available() and R.has_models():
            R.set_threads(cpu_info()["nproc"])
            t0 = time.perf_counter()
            job = R.GnnJob(N, V, E, 4)
            ref_rounds = [job.run()[:N].copy()]
            p_ref = job.p[:N].copy()
            for _ in range(9):
                ref_rounds.append(job.culberson()[:N].copy())
            job.close()
            ref_s = time.perf_counter() - t0
            eq = [bool(np.array_equal(a, b)) for a, b in zip(rounds, ref_rounds)]
            p_eq = bool(np.array_equal(p_gpu.view(np.uint64), p_ref.view(np.uint64)))
            entry["parity"] = {"checked": True, "against": "reference gnn_internal_par + 9 x (p := color, "
                                                            "jones_plassmann_internal), oracle/_ref",
                               "p_bits_equal": p_eq, "colors_equal_per_round": eq,
                               "colors_per_round": [int(c.max()) for c in rounds],
                               "colors_per_round_reference": [int(c.max()) for c in ref_rounds],
                               "all_equal": p_eq and all(eq), "reference_s_incl_setup": ref_s}
        else:
            entry["parity"] = {"checked": False, "why": "reference not built"}
        out[key] = entry
        del V, E
    for m in models.values():
        m.close()
    ctx.close()
    return out


# ---- batched vs plain: many independent graphs in one launch ------------------------------------

def run_batched(args, device):
    """4,096 mixed graphs (n log-uniform in [1e3, 2e5]; even seeds Erdos-Renyi with average degree
    U[8, 32], odd seeds R-MAT with edge factor 8; seeds 1000..5095) colored by GNN2 and by LF: one
    autotuned, CUDA-graph-captured gc_batch_color pass over the device-resident segmented CSR against
    one plain gc_priority + gc_color per graph (graphs device-resident too).  Both legs return each
    graph's color count to the host; colors are compared vertex by vertex."""
    import gnn_coloring as gcn
    G = args.batch_graphs
    t0 = time.perf_counter()
    voff, V, E = gcn.gen_mixed_batch(G, 1000, 1000, 200000)
    gen_s = time.perf_counter() - t0
    N, M = int(voff[G]), int(V[int(voff[G])])
    ctx = gcn.Context(device)
    model = _model(ctx, gcn, 2)
    heurs = [("GNN2", "GNN", model), ("LF", "LF", None)]
    out = {"workload": f"{G} mixed graphs: n log-uniform [1000, 200000]; even seeds Erdos-Renyi avg degree "
                       f"U[8,32], odd seeds R-MAT ef 8; seeds 1000..{999 + G}",
           "G": G, "N": N, "M": M, "model": model_desc(2), "host_generation_s": gen_s, "heuristics": {}}
    b = gcn.Batch(ctx, voff, V, E)
    batch_colors = {}
    for name, h, m in heurs:
        tuning, tuned_ms = b.autotune(h, m, 0, effort=1)
        counts = b.color(h, m)          # first call runs directly and captures the pipeline
        ctx.sync()
        reps = max(3, min(args.steps, 10))
        t0 = time.perf_counter()
        for _ in range(reps):
            counts = b.color(h, m)      # one cudaGraphLaunch, per-graph counts read back
        batch_s = (time.perf_counter() - t0) / reps
        batch_colors[name] = (b.colors(), counts.copy())
        out["heuristics"][name] = {"batched_ms": 1e3 * batch_s, "batched_edges_per_s": M / batch_s,
                                   "autotuned": tuning.as_dict(), "autotune_best_ms": tuned_ms}
    b.close()
    # plain leg: the same graphs, one device-resident gc_graph each, one priority + color per graph
    graphs = []
    for g in range(G):
        a, z = int(voff[g]), int(voff[g + 1])
        ea, ez = int(V[a]), int(V[z])
        graphs.append(gcn.Graph(ctx, z - a, (V[a:z + 1] - V[a]).astype(np.uint32), E[ea:ez]))
    for name, h, m in heurs:
        # one untimed call per graph first: each graph's lazily allocated buffers (and, for the GNN,
        # its feature-row order) exist before the timed pass, so that pass times launches and work
        for gr in graphs:
            gr.priority(h, m)
            gr.color()
        ctx.sync()
        counts = np.zeros(G, np.int64)
        t0 = time.perf_counter()
        for i, gr in enumerate(graphs):
            gr.priority(h, m)
            counts[i] = gr.color()      # the color count, read back per graph
        plain_s = time.perf_counter() - t0
        bc, bcounts = batch_colors[name]
        same = bool(np.array_equal(counts, bcounts))
        for i, gr in enumerate(graphs):
            if not same:
                break
            same = np.array_equal(gr.colors(), bc[int(voff[i]):int(voff[i + 1])])
        r = out["heuristics"][name]
        r.update({"plain_ms": 1e3 * plain_s, "plain_edges_per_s": M / plain_s,
                  "speedup": plain_s / (r["batched_ms"] / 1e3), "colors_identical": same})
    for gr in graphs:
        gr.close()
    model.close()
    ctx.close()
    return out


# ---- serving: open-loop arrivals of mixed jobs ----------------------------------------------------

SERVE_RATES = (100, 1000, 5000, 20000)


def serving_pool(seed: int = 5):
    """Graphs the jobs draw from: 48 Erdos-Renyi (n uniform in [1000, 50000], average degree 16),
    2 R-MAT scale 20 and 1 R-MAT scale 24 (edge factor 16, a/b/c = 0.57/0.19/0.19)."""
    import gnn_coloring as gcn
    rng = np.random.default_rng(seed)
    small = []
    for i in range(48):
        n = int(rng.integers(1000, 50001))
        small.append(gcn.gen_er(n, 8 * n, 10_000 + i))
    medium = [gcn.gen_rmat(1 << 20, 16, 20 + i) for i in range(2)]
    large = [gcn.gen_rmat(1 << 24, 16, 24)]
    return small, medium, large


def serving_jobs(pool, J: int, seed: int):
    """J jobs: 90% small, 9% medium, 1% large graphs; heuristic uniform over FF, LLF, GNN3."""
    small, medium, large = pool
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(J):
        r = rng.random()
        cls = small if r < 0.90 else (medium if r < 0.99 else large)
        k = int(rng.integers(len(cls)))
        jobs.append((cls[k], ("FF", "LLF", "GNN")[int(rng.integers(3))]))
    return jobs


def _sweep(srv, pool, J, replay, alone_counts):
    """Poisson arrivals at each rate of SERVE_RATES (J jobs, more at high rates: up to 2 s of arrivals,
    at most 1,500) through `replay`; per-rate latency percentiles and throughput from the server's
    own statistics."""
    sweep, same = [], True
    for i, rate in enumerate(SERVE_RATES):
        Jr = max(J, min(1500, 2 * rate))  # enough large jobs at the high rates for a stable edges/s
        jobs = serving_jobs(pool, Jr, 1000 + i)
        arrive = np.cumsum(np.random.default_rng(2000 + i).exponential(1.0 / rate, Jr))
        srv.reset_stats()
        infos = replay(arrive, jobs)
        st = srv.stats()
        for (gr, h), inf in zip(jobs, infos):
            c = alone_counts.get((id(gr), h))
            if c is not None and c != inf["colors"]:
                same = False
        by_class = {}
        for cls, lo, hi in (("small", 0, 1 << 17), ("rmat20", 1 << 17, 1 << 21), ("rmat24", 1 << 21, 1 << 32)):
            lat = [inf["latency_ms"] for inf in infos if lo < inf["N"] + 1 <= hi]
            if lat:
                by_class[cls] = {"jobs": len(lat), "p50_ms": float(np.percentile(lat, 50)),
                                 "p99_ms": float(np.percentile(lat, 99))}
        sweep.append({"offered_jobs_per_s": rate, "jobs": Jr, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                      "by_size": by_class,
                      "max_ms": st["max_ms"], "edges_per_s": st["edges_per_s"],
                      "jobs_per_s": st["completed"] / st["span_s"] if st["span_s"] else None,
                      "passes": st["launches"], "batched_jobs": st["batched_jobs"],
                      "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9, "pool_peak_gb": st["pool_peak_bytes"] / 1e9})
    return sweep, same


def _plain_sequential(jobs, run_one, warm=False):
    """The same jobs one after another through the plain path: throughput and per-job latency.  With
    `warm`, every job runs once untimed first, so that graphs that stay resident have their lazily
    allocated buffers before the timed pass."""
    lat, edges = [], 0
    counts = {}
    if warm:
        for gr, h in jobs:
            run_one(gr, h)
    t0 = time.perf_counter()
    for gr, h in jobs:
        ta = time.perf_counter()
        counts[(id(gr), h)] = run_one(gr, h)
        lat.append(1e3 * (time.perf_counter() - ta))
        edges += int(gr[1][-1])
    dt = time.perf_counter() - t0
    return ({"jobs": len(jobs), "edges_per_s": edges / dt, "jobs_per_s": len(jobs) / dt,
             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}, counts)


def run_serving(args, device):
    """The serving mix in two forms: jobs bringing their CSR in host memory (uploaded per job), and
    jobs on CSRs registered once (device-resident).  Each against the same jobs run one at a time
    through the plain path in the same form."""
    import gnn_coloring as gcn
    t0 = time.perf_counter()
    pool = serving_pool()
    gen_s = time.perf_counter() - t0
    params3, md3 = gcn.model_read(model_file(3)) if model_file(3) else gcn.synthetic_model(3, MODEL_SEED)
    J = args.serve_jobs
    base_jobs = serving_jobs(pool, J, 99)
    ctx = gcn.Context(device)
    model = gcn.Model(ctx, params3, md3)

    def host_one(gr, h):
        g = gcn.Graph(ctx, *gr)
        g.priority(h, model if h == "GNN" else None)
        c = g.color()
        g.colors()
        g.close()
        return c

    plain_host, counts = _plain_sequential(base_jobs, host_one)
    resident = {id(gr): gcn.Graph(ctx, *gr) for cls in pool for gr in cls}

    def resident_one(gr, h):
        g = resident[id(gr)]
        g.priority(h, model if h == "GNN" else None)
        c = g.color()
        g.colors()
        return c

    plain_res, counts_res = _plain_sequential(base_jobs, resident_one, warm=True)
    counts.update(counts_res)
    for g in resident.values():
        g.close()
    model.close()
    ctx.close()

    srv = gcn.Server(device=device, models=[(params3, md3)])
    lanes = int(gcn.serve_config_default().lanes)

    def replay_host(arrive, jobs):
        return srv.replay(arrive, [gr for gr, _ in jobs], [h for _, h in jobs],
                          layers=[3 if h == "GNN" else 0 for _, h in jobs])[1]

    sweep_host, same1 = _sweep(srv, pool, J, replay_host, counts)
    reg = {id(gr): srv.register(*gr) for cls in pool for gr in cls}

    def replay_res(arrive, jobs):
        return srv.replay_registered(arrive, [reg[id(gr)] for gr, _ in jobs], [h for _, h in jobs],
                                     layers=[3 if h == "GNN" else 0 for _, h in jobs])[1]

    sweep_res, same2 = _sweep(srv, pool, J, replay_res, counts)
    srv.close()

    def form(plain, sweep):
        best = max(sweep, key=lambda r: r["edges_per_s"])
        best_j = max(r["jobs_per_s"] or 0 for r in sweep)
        return {"plain_sequential": plain, "sweep": sweep,
                "speedup_edges_per_s": best["edges_per_s"] / plain["edges_per_s"],
                "speedup_jobs_per_s": best_j / plain["jobs_per_s"]}

    return {"mix": "90% Erdos-Renyi n in [1000, 50000] avg degree 16, 9% R-MAT scale 20, 1% R-MAT scale 24 "
                   "(ef 16); heuristic uniform over FF, LLF, GNN3; open-loop Poisson arrivals",
            "pool_generation_s": gen_s, "jobs_per_rate": J, "lanes": lanes,
            "host_csr": form(plain_host, sweep_host), "resident_csr": form(plain_res, sweep_res),
            "color_counts_identical_to_alone": same1 and same2}


def run_e2e(args, N, V, E, torch):
    import gnn_coloring as gcn
    M = int(V[N])
    if model_file(3):
        os.environ["GC_MODEL_DIR"] = REF_MODELS
    else:
        work = tempfile.mkdtemp(prefix="gnne2e_")
        gcn.model_write(os.path.join(work, "m3.gnn"), *gcn.synthetic_model(3, MODEL_SEED))
        os.environ["GC_MODEL_DIR"] = work
    os.environ["GC_DEVICE"] = str(torch.cuda.current_device())
    lib = gcn.lib
    C.c_int.in_dll(lib, "layers").value = 3
    lib.gnn_setup.argtypes = [C.c_uint32, C.c_uint32]
    lib.gnn_setup.restype = C.c_void_p
    lib.jones_plassmann_setup.argtypes = [C.c_uint32, C.c_uint32]
    lib.jones_plassmann_setup.restype = C.c_void_p
    lib.gnn_internal_par.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
    lib.gnn_cleanup.argtypes = [C.c_void_p]
    lib.jones_plassmann_cleanup.argtypes = [C.c_void_p]
    ad = lib.gnn_setup(N, M)
    jp = lib.jones_plassmann_setup(N, M)
    hV = torch.from_numpy(np.ascontiguousarray(V).view(np.int32)).pin_memory()
    hE = torch.from_numpy(np.ascontiguousarray(E).view(np.int32)).pin_memory()
    hp = torch.empty(N + 8, dtype=torch.float64).pin_memory()
    hc = torch.empty(N, dtype=torch.int32).pin_memory()

    def call():
        lib.gnn_internal_par(N, hV.data_ptr(), hE.data_ptr(), ad, jp, hp.data_ptr(), hc.data_ptr())

    for _ in range(max(3, args.warmup)):
        call()
    steps = max(1, args.steps)
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    dt = time.perf_counter() - t0
    lib.gnn_cleanup(ad)
    lib.jones_plassmann_cleanup(jp)
    return {"value": M * steps / dt, "unit": UNIT, "h2d_bytes_per_step": 4 * (N + 1) + 4 * M,
            "d2h_bytes_per_step": 8 * N + 4 * N, "ms_per_step": 1e3 * dt / steps,
            "entry_point": "gnn_internal_par (include/gnn.h) from pinned host memory"}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="rmat22", choices=["rmat22", "rmat18", "er65k"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the ER-65k and mesh-graph measurements")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving sweep")
    ap.add_argument("--batch-graphs", type=int, default=4096)
    ap.add_argument("--serve-jobs", type=int, default=300)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
