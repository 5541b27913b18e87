#!/usr/bin/env python
"""Benchmark: batched grid-kNN queries/s at K=16 on one B200.

Workload (BASELINE configuration "batched uneven sizes"): 16 synthetic
clouds, room-like and LiDAR-like alternately, point counts log-uniform in
[20k, 200k] (1.464M points), offset-concatenated, self query, K=16, 5 cm
voxels, parent cell = 4 voxels.  One step = one pass of the whole path over
the batch: grid construction + candidate gather + top-K + remap, replayed
from a CUDA graph, inputs already in HBM.  L2 is flushed (256 MiB memset)
before every timed step, outside its events.

Also reported on the same line: ``e2e`` (the public ``knn_query`` call with
host buffers, H2D and D2H inside the timed region), the loop of plain
per-cloud calls, forward+backward and backward-only time, the backward's
error against FP64 finite differences, the query kernel's roofline,
recall@K against an FP64 brute force (timed), and the reference's CPU kNN
(nanoflann) timed on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--k 16]
Under torchrun every rank takes a share of the clouds (whole clouds, largest
first onto the least-loaded rank); there is no collective in the data path.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--k", type=int, default=16)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the per-cloud, fwd+bwd and CPU-baseline legs")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer e2e leg")
    ap.add_argument("--small-rows", action="store_true",
                    help="only the uniform-cube and hierarchy rows (profiling)")
    ap.add_argument("--rows-only", action="store_true",
                    help="only the per-path rows and one distance backward (profiling)")
    ap.add_argument("--no-tune", action="store_true",
                    help="default launch shape instead of the autotuned one")
    ap.add_argument("--clouds", type=int, default=16,
                    help="use the first N clouds of the batch (small cases for profiling)")
    return ap.parse_args()


# ----------------------------------------------------------------- helpers

def shard_clouds(counts, world):
    """Greedy longest-first assignment of whole clouds to ranks."""
    load = [0] * world
    owner = [0] * len(counts)
    for c in sorted(range(len(counts)), key=lambda i: -int(counts[i])):
        r = min(range(world), key=lambda j: load[j])
        owner[c] = r
        load[r] += int(counts[c])
    return owner


def take_clouds(batch, ids):
    starts = np.concatenate([[0], batch.offsets[:-1]])
    parts = [batch.xyz[starts[i]:batch.offsets[i]] for i in ids]
    counts = np.array([len(p) for p in parts], np.int64)
    xyz = np.ascontiguousarray(np.concatenate(parts)) if parts else np.zeros((0, 3), np.float32)
    return xyz, np.cumsum(counts)


class ClockSampler:
    """NVML samples of the SM clock and throttle reasons while the timed
    region runs (a polling thread, 1 ms period)."""

    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, device_index):
        self.device_index = device_index
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self.err = None

    def __enter__(self):
        self._stop = threading.Event()
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.device_index).uuid)
            try:
                h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except pynvml.NVMLError:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self._h, self._nv = h, pynvml
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception as exc:  # sampling is best effort; recorded in the output
            self.err = f"{type(exc).__name__}: {exc}"[:120]
            self._h = None
        return self

    def _poll(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.sm.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for name, mask in self.REASONS.items():
                    if bits & mask:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.001)

    def __exit__(self, *exc):
        self._stop.set()
        if getattr(self, "_h", None) is not None:
            self.thread.join(timeout=2)

    def summary(self):
        out = {"sm_mhz": statistics.median(self.sm) if self.sm else None,
               "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
               "samples": len(self.sm)}
        if self.err:
            out["error"] = self.err
        return out


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _query_profile(k):
    path = os.path.join(ROOT, "profiles", f"k_query_uneven_batch_k{k}.txt")
    if not os.path.exists(path):
        return None, None
    with open(path) as f:
        return os.path.relpath(path, ROOT), f.read()


def profiled_traffic(k):
    """DRAM bytes (read + write) of one query-kernel launch on this workload,
    from the committed ncu summary of that kernel; None when absent."""
    import re
    _, text = _query_profile(k)
    m = re.search(r"dram_bytes_per_launch\s*=\s*([0-9]+)", text or "")
    return int(m.group(1)) if m else None


def profiled_limiter(k):
    """The unit that bounds the query kernel, from the same ncu summary: the
    kernel is instruction-bound (ALU pipe), so the HBM fraction alone does
    not describe it."""
    import re
    path, text = _query_profile(k)
    if text is None:
        return None
    alu = re.search(r"sm__inst_executed_pipe_alu \(active\)\s+([0-9.]+) %", text)
    issue = re.search(r"smsp__issue_active \(active\)\s+([0-9.]+) %", text)
    per_q = re.search(r"~([0-9]+) warp instructions per query", text)
    if not (alu and issue and per_q):
        return None
    return {"unit": "ALU pipe (integer compare/select)",
            "alu_pipe_active_pct": float(alu.group(1)),
            "issue_active_pct": float(issue.group(1)),
            "warp_instructions_per_query": int(per_q.group(1)),
            "source": path}


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_oracle_rate(xyz, offsets, k, voxel, budget_s=20.0):
    """The oracle (C restatement of the reference path, OpenMP on every host
    core) on a bounded sample: whole clouds, largest prefix of the batch that
    fits the time budget after one probe run on the first cloud."""
    from oracle import oracle as O
    cores = cpu_cores()
    starts = np.concatenate([[0], offsets[:-1]])
    t0 = time.perf_counter()
    O.knn_offsets(xyz[: offsets[0]], offsets[:1], k, voxel, 2, nthreads=cores)
    per_point = (time.perf_counter() - t0) / max(int(offsets[0]), 1)
    take = 1
    while take < len(offsets) and per_point * offsets[take] < budget_s * 0.5:
        take += 1
    sub_xyz = xyz[: offsets[take - 1]]
    sub_off = offsets[:take]
    t0 = time.perf_counter()
    O.knn_offsets(sub_xyz, sub_off, k, voxel, 2, nthreads=cores)
    dt = time.perf_counter() - t0
    n = int(sub_off[-1])
    return {"value": n / dt, "unit": "queries/s", "cores": cores, "kind": "port",
            "sample": f"first {take} of {len(offsets)} clouds ({n} points, construction + "
                      f"query), one pass, OpenMP x{cores}", "seconds": dt}


def nanoflann_rate(batch, k, steps, warmup):
    """The reference's CPU kNN (nanoflann, built from the reference's header
    into oracle/_ref) over the whole batch on every host core: queries/s of
    KD-tree construction + exact top-K, one pass over the batch per step."""
    from oracle import ref_nanoflann
    cores = cpu_cores()
    n = int(len(batch.xyz))
    for _ in range(warmup):
        ref_nanoflann.knn(batch.xyz, batch.offsets, k, nthreads=cores)
    secs = []
    for _ in range(steps):
        _, _, tb, tq = ref_nanoflann.knn(batch.xyz, batch.offsets, k, nthreads=cores)
        secs.append(tb + tq)
    return {"value": n * len(secs) / sum(secs), "unit": "queries/s", "cores": cores,
            "kind": "reference", "ms_per_step": sum(secs) / len(secs) * 1e3,
            "sample": f"whole batch ({n} points, {len(batch.offsets)} clouds) x {steps} passes: "
                      f"nanoflann KD-tree build (leaf 20) + exact K={k} query, OpenMP x{cores}"}


# --------------------------------------------------------------- our arm

def run_ours(args, rank, world, local_rank, dist):
    import torch

    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200 import _lib, synthetic

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    k = args.k
    batch = synthetic.uneven_batch()
    if args.clouds < len(batch.counts):
        batch = synthetic.first_clouds(batch, args.clouds)
    voxel = synthetic.C4_VOXEL
    # Weak scaling: the job is `world` copies of the 16-cloud batch; whole
    # clouds are assigned to ranks, largest first onto the least-loaded rank.
    job_counts = np.tile(batch.counts, world)
    owner = shard_clouds(job_counts, world)
    mine = [c % len(batch.counts) for c in range(len(job_counts)) if owner[c] == rank]
    xyz_h, off_h = take_clouds(batch, mine)
    n = len(xyz_h)
    xyz = torch.from_numpy(xyz_h).to(dev)
    off = torch.from_numpy(off_h).to(dev)
    lib = _lib.load()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    # --- launch shape picked by the autotuner on this workload (untimed)
    from flashknn_exprepo_b200 import autotune
    cfg = None if args.no_tune else autotune.tune_offsets(xyz, off, k, voxel, 2)
    tuned = autotune.last_results() if cfg is not None else {}

    # --- capture the batched pipeline in a CUDA graph
    stream = torch.cuda.Stream(dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(stream):
        fk.ops.knn_offsets(xyz, off, k, voxel, 2, config=cfg)  # workspace sized, kernels loaded
        torch.cuda.synchronize(dev)
        launches_per_step = fk.ops.last_launch_count()
        lib.fknn_profile_enable(1)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            idx_g, dist_g = fk.ops.knn_offsets(xyz, off, k, voxel, 2, config=cfg)
    torch.cuda.current_stream(dev).wait_stream(stream)
    torch.cuda.synchronize(dev)

    prof_buf = ctypes_float_array(1)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    step_ms, kern_ms = [], []
    with ClockSampler(local_rank) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            graph.replay()
            e1.record()
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            if lib.fknn_profile_read(ctypes.cast(prof_buf, ctypes.c_void_p), 1) == 1:
                kern_ms.append(prof_buf[0])
    torch.cuda.synchronize(dev)
    lib.fknn_profile_enable(0)
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        q = torch.tensor([n], dtype=torch.int64, device=dev)
        dist.all_reduce(q)
        total_queries = int(q.item())
        dist.barrier()
    else:
        total_queries = n
    value = total_queries * args.steps / (total_ms / 1e3)

    # parity of the timed graph against a fresh eager call
    ei, ed = fk.ops.knn_offsets(xyz, off, k, voxel, 2, config=cfg, validate=True)
    graph_matches = bool(torch.equal(ei, idx_g) and torch.equal(ed, dist_g))

    out = {"value": value, "ms_per_step": total_ms / args.steps, "n_points": total_queries,
           "clocks": clocks.summary(), "kernel_ms": kern_ms, "launches_per_step": launches_per_step,
           "graph_matches_eager": graph_matches, "local_n": n,
           "launch_shape": None if cfg is None else {
               "warps_per_cta": cfg.warps_per_cta, "tile_records": cfg.tile_records,
               "min_candidates_per_lane": cfg.min_candidates_per_lane,
               "staging_depth": cfg.staging_depth,
               "tuned": next(iter(tuned.values()), None)}}
    del graph

    if args.no_e2e:
        out["e2e"] = None
        return out

    # --- e2e through the public API: pinned host in, pinned host out
    xyz_pin = torch.from_numpy(xyz_h).pin_memory()
    off_pin = torch.from_numpy(off_h).pin_memory()
    idx_pin = torch.empty((n, k), dtype=torch.int32).pin_memory()
    dist_pin = torch.empty((n, k), dtype=torch.float32).pin_memory()

    def single_call():
        x = xyz_pin.to(dev, non_blocking=True)
        o = off_pin.to(dev, non_blocking=True)
        i, d = fk.knn_query(k, x, o, voxel_size=voxel, num_down=2)
        idx_pin.copy_(i, non_blocking=True)
        dist_pin.copy_(d, non_blocking=True)

    def host_call():
        fk.knn_query_host(k, xyz_pin, off_pin, idx_pin, dist_pin, voxel_size=voxel,
                          num_down=2, config=cfg)

    def timed(step):
        for _ in range(max(2, args.warmup)):
            step()
        torch.cuda.synchronize(dev)
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return sum(ms)

    single_total = timed(single_call)
    e2e_total = timed(host_call)
    if world > 1:
        t = torch.tensor([e2e_total], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    out["e2e"] = {"value": total_queries * args.steps / (e2e_total / 1e3), "unit": "queries/s",
                  "h2d_bytes_per_step": int(xyz_pin.numel() * 4 + off_pin.numel() * 8),
                  "d2h_bytes_per_step": int(n * k * 8),
                  "call": "knn_query_host: pinned host in/out, copies overlapped with the "
                          "query in 8 whole-cloud runs",
                  "single_call": {"value": n * args.steps / (single_total / 1e3),
                                  "unit": "queries/s",
                                  "call": "H2D, knn_query, D2H of idx and dist, one after "
                                          "the other"}}

    if not args.no_extras and world == 1:
        out.update(extras_single_gpu(args, fk, torch, dev, batch, voxel, flush))
    return out


def ctypes_float_array(n):
    return (ctypes.c_float * n)()


def extras_single_gpu(args, fk, torch, dev, batch, voxel, flush):
    """Per-cloud loop, forward+backward, recall sample (rank 0, N=1)."""
    from flashknn_exprepo_b200 import synthetic
    k = args.k
    res = {}
    starts = np.concatenate([[0], batch.offsets[:-1]])
    clouds = [torch.from_numpy(batch.xyz[s:e]).to(dev) for s, e in zip(starts, batch.offsets)]
    offs = [torch.tensor([len(c)], dtype=torch.int64, device=dev) for c in clouds]

    def per_cloud():
        for c, o in zip(clouds, offs):
            fk.ops.knn_offsets(c, o, k, voxel, 2)

    for _ in range(2):
        per_cloud()
    torch.cuda.synchronize(dev)
    reps = max(3, args.steps // 4)
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        per_cloud()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    n = len(batch.xyz)
    res["per_cloud"] = {"value": n * reps / (sum(ms) / 1e3), "unit": "queries/s",
                        "ms_per_step": sum(ms) / reps,
                        "what": "loop of 16 plain fknn_knn_offsets calls, one per cloud, eager"}
    # the same loop captured in one CUDA graph: no host launch overhead, so
    # the comparison with the batched step is launch model against launch model
    stream = torch.cuda.Stream(dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(stream):
        per_cloud()  # workspace of this stream sized for the largest cloud
        torch.cuda.synchronize(dev)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            per_cloud()
    torch.cuda.current_stream(dev).wait_stream(stream)
    torch.cuda.synchronize(dev)
    gms = _event_ms(torch, graph.replay, flush, reps=reps)
    del graph
    res["per_cloud_graph"] = {"value": n / (gms * 1e-3), "unit": "queries/s", "ms_per_step": gms,
                              "what": "the same 16 per-cloud calls replayed from one CUDA graph"}

    # the batched step at K=32 (the batch configuration's second K): one
    # graph of construction + query, replayed, L2 flushed before each
    xyz_all = torch.from_numpy(batch.xyz).to(dev)
    off_all = torch.from_numpy(batch.offsets).to(dev)
    with torch.cuda.stream(stream):
        fk.ops.knn_offsets(xyz_all, off_all, 32, voxel, 2)
        torch.cuda.synchronize(dev)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            fk.ops.knn_offsets(xyz_all, off_all, 32, voxel, 2)
    torch.cuda.current_stream(dev).wait_stream(stream)
    torch.cuda.synchronize(dev)
    kms = _event_ms(torch, graph.replay, flush, reps=reps)
    del graph
    res["batched_k32"] = {"value": n / (kms * 1e-3), "unit": "queries/s", "ms_per_step": kms,
                          "what": "batched construction + query at K=32, one CUDA graph"}

    # forward + backward (loss = sum(w * d), w ~ N(0,1))
    xyz = torch.from_numpy(batch.xyz).to(dev)
    off = torch.from_numpy(batch.offsets).to(dev)
    w = torch.from_numpy(synthetic.backward_weights(n, k)).to(dev)

    def fwd_bwd():
        x = xyz.detach().requires_grad_(True)
        _, d = fk.knn_query(k, x, off, voxel_size=voxel, num_down=2)
        (w * d.masked_fill(~torch.isfinite(d), 0)).sum().backward()
        return x.grad

    for _ in range(2):
        fwd_bwd()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fwd_bwd()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    res["fwd_bwd_ms"] = sum(ms) / reps

    # the backward kernels alone, on the forward's outputs
    x = xyz.detach()
    idx, d = fk.ops.knn_offsets(x, off, k, voxel, 2)
    g = w * torch.isfinite(d).to(w.dtype)
    grad = torch.empty_like(x)
    for _ in range(2):
        fk.ops.backward(x, x, idx, d, g, grad_q=grad, grad_p=grad, accumulate=True)
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        flush.zero_()
        grad.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fk.ops.backward(x, x, idx, d, g, grad_q=grad, grad_p=grad, accumulate=True)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    res["backward_ms"] = sum(ms) / reps
    res["fd_check"] = fd_check(fk, torch, dev, batch, k, voxel)
    res["recall"] = fp64_recall(batch, idx.cpu().numpy(), k)
    res["rows"] = rows_single_gpu(fk, torch, dev, flush, measured_peak_hbm()[0])
    return res


def _event_ms(torch, fn, flush, reps=5):
    """Mean device ms of fn over reps, L2 flushed before each, after 2 warm-ups."""
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / reps


def row_hierarchy(fk, torch, dev):
    """The DeLA hierarchy builder (4 levels, K=24, alpha 16) on the
    voxel-first LiDAR scan: wall clock of one call, mean of 3."""
    from flashknn_exprepo_b200 import hierarchy, synthetic
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    lid = T(synthetic.lidar(dedup=True))
    hierarchy.build_flash_hierarchy(lid)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        hierarchy.build_flash_hierarchy(lid)
    torch.cuda.synchronize()
    return {"value": (time.perf_counter() - t0) / 3 * 1e3, "unit": "ms",
            "n_points": int(lid.shape[0]),
            "what": "wall clock incl. one count read-back per level"}


def row_cube(fk, torch, dev, flush):
    """The uniform cube (16,384 points, K=16): one self-query call, eager and
    replayed from its cached CUDA graph."""
    from flashknn_exprepo_b200 import synthetic
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    cube = T(synthetic.uniform_cube())
    co = torch.tensor([cube.shape[0]], device=dev)
    ms = _event_ms(torch, lambda: fk.ops.knn_offsets(cube, co, 16, synthetic.C1_VOXEL, 2), flush)
    gms = _event_ms(torch, lambda: fk.ops.knn_offsets(cube, co, 16, synthetic.C1_VOXEL, 2,
                                                      graph=True), flush)
    return {"value": cube.shape[0] / (ms * 1e-3), "unit": "queries/s",
            "ms": ms, "n_points": int(cube.shape[0]), "graph_ms": gms,
            "graph": "the same call with graph=True (a cached CUDA graph of the pipeline "
                     "replayed)"}


def rows_single_gpu(fk, torch, dev, flush, peak_gbs, clouds=16):
    """The paths around the batched query, each on its own workload:
    adaptive-neighbourhood query (LiDAR scan), back query and voxel-first
    subsampling (16-cloud batch), the DeLA hierarchy builder (LiDAR scan),
    radius-limited query (room), the room at K=32 through the self query,
    the selected query (every 4th point) and the reference table ABI, the
    uniform cube at K=16, the LiDAR scan at alpha 4 and 8, and neighbour
    feature grouping (16-cloud batch, 64 channels, forward with its HBM
    roofline, and backward)."""
    from flashknn_exprepo_b200 import synthetic
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    rows = {}
    # adaptive neighbourhood, LiDAR scan ~118k points, K=16
    lidar = synthetic.lidar()
    grid = T(np.floor(lidar / np.float32(synthetic.C3_VOXEL)).astype(np.int64))
    lx = T(lidar)
    eager = _event_ms(torch, lambda: fk.ops.adaptive_query(grid, None, 16, xyz=lx), flush)
    stream = torch.cuda.Stream(dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(stream):
        fk.ops.adaptive_query(grid, None, 16, xyz=lx)   # workspace sized on this stream
        torch.cuda.synchronize(dev)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            fk.ops.adaptive_query(grid, None, 16, xyz=lx)
    torch.cuda.current_stream(dev).wait_stream(stream)
    torch.cuda.synchronize(dev)
    ms = _event_ms(torch, graph.replay, flush)
    del graph
    lib = fk._lib.load()
    lib.fknn_profile_enable(1)
    buf = ctypes_float_array(1)
    qms = []
    for _ in range(5):
        flush.zero_()
        fk.ops.adaptive_query(grid, None, 16, xyz=lx)
        torch.cuda.synchronize()
        if lib.fknn_profile_read(ctypes.cast(buf, ctypes.c_void_p), 1) == 1:
            qms.append(buf[0])
    lib.fknn_profile_enable(0)
    _, _, lv = fk.ops.adaptive_query(grid, None, 16, xyz=lx, want_levels=True)
    lvl, cnt = torch.unique(lv, return_counts=True)
    rows["adaptive_lidar_k16"] = {"value": len(lidar) / (ms * 1e-3), "unit": "queries/s",
                                  "ms": ms, "eager_ms": eager, "n_points": len(lidar),
                                  "query_kernel_ms": statistics.median(qms) if qms else None,
                                  "points_per_level": {int(a): int(b) for a, b in
                                                       zip(lvl.tolist(), cnt.tolist())},
                                  "step": "CUDA-graph replay of the whole adaptive pipeline"}
    # back query K=1 and voxel-first subsampling, 16-cloud batch (or its
    # first `clouds` clouds: smaller cases for profiling)
    b = synthetic.uneven_batch()
    if clouds < len(b.counts):
        b = synthetic.first_clouds(b, clouds)
    bx = T(b.xyz)
    bb = T(np.repeat(np.arange(len(b.counts)), b.counts).astype(np.int64))
    ms = _event_ms(torch, lambda: fk.ops.voxel_first(bx, 0.1, bb), flush)
    rows["voxel_first_batch"] = {"value": len(b.xyz) / (ms * 1e-3), "unit": "points/s",
                                 "ms": ms, "voxel_m": 0.1}
    sel = fk.ops.voxel_first(bx, 0.1, bb)
    ms = _event_ms(torch, lambda: fk.ops.back_query(bx, sel, 0.2, 1, bb), flush)
    rows["back_query_batch_k1"] = {"value": len(b.xyz) / (ms * 1e-3), "unit": "queries/s",
                                   "ms": ms, "subset_points": int(sel.numel()),
                                   "query_grid_m": 0.2}
    rows["hierarchy_lidar"] = row_hierarchy(fk, torch, dev)
    # radius-limited query, room ~80k points, K=32, r=0.1 m
    room = T(synthetic.room())
    ro = torch.tensor([room.shape[0]], device=dev)
    ms = _event_ms(torch, lambda: fk.ops.ball_query_offsets(room, ro, 32, 0.1, 0.025, 2), flush)
    rows["ball_query_room_k32"] = {"value": room.shape[0] / (ms * 1e-3), "unit": "queries/s",
                                   "ms": ms, "radius_m": 0.1}
    # room (C2), K=32, 4 cm voxels, alpha 4: every point, the stride-4 subset
    # (selected query), and the reference table ABI (tables built once by
    # fknn_build_tables, which reads the parent count back; query timed alone)
    rgrid = torch.floor(room / synthetic.C2_VOXEL).long()
    ms = _event_ms(torch, lambda: fk.ops.knn_grid(room, rgrid, None, 32, 2), flush)
    rows["self_query_room_k32"] = {"value": room.shape[0] / (ms * 1e-3), "unit": "queries/s",
                                   "ms": ms, "n_points": int(room.shape[0])}
    qi = torch.arange(0, room.shape[0], 4, device=dev)
    ms = _event_ms(torch, lambda: fk.ops.knn_grid(room, rgrid, None, 32, 2, query_indices=qi),
                   flush)
    rows["selected_query_room_k32"] = {"value": qi.numel() / (ms * 1e-3), "unit": "queries/s",
                                       "ms": ms, "n_queries": int(qi.numel()),
                                       "n_support": int(room.shape[0])}
    bms = _event_ms(torch, lambda: fk.ops.build_tables(rgrid, None, 2), flush)
    tb = fk.ops.build_tables(rgrid, None, 2)
    xs = room[tb["order"]].contiguous()
    ms = _event_ms(torch, lambda: fk.ops.query_tables(xs, tb["steps"], tb["neigh"], tb["cnt"],
                                                      32), flush)
    rows["query_tables_room_k32"] = {"value": room.shape[0] / (ms * 1e-3), "unit": "queries/s",
                                     "ms": ms, "build_tables_ms": bms,
                                     "what": "reference table ABI (FlashKNN_Query_Dynamic_Load "
                                             "boundary): query on caller-built tables"}
    # the largest cloud of the uneven batch through the table ABI at K=16
    # (tables from fknn_build_tables, equal to the reference's own; the
    # reference arm times FlashKNN_Query_Dynamic_Load on them)
    c = int(np.argmax(b.counts))
    lx_ = T(b.xyz[int(b.offsets[c] - b.counts[c]):int(b.offsets[c])])
    lgrid = torch.floor(lx_ * (1.0 / synthetic.C4_VOXEL)).long()
    ltb = fk.ops.build_tables(lgrid, None, 2)
    lxs = lx_[ltb["order"]].contiguous()
    ms = _event_ms(torch, lambda: fk.ops.query_tables(lxs, ltb["steps"], ltb["neigh"],
                                                      ltb["cnt"], 16), flush)
    rows["query_tables_largest_cloud_k16"] = {
        "value": lx_.shape[0] / (ms * 1e-3), "unit": "queries/s", "ms": ms,
        "n_points": int(lx_.shape[0]),
        "what": "reference table ABI on the largest cloud of the uneven batch"}
    # the same stride-4 queries through the selected-query table ABI: qindex =
    # their sorted positions grouped by parent, steps_query = per-parent offsets
    inv = torch.empty_like(tb["order"])
    inv[tb["order"]] = torch.arange(room.shape[0], device=dev)
    qpos = inv[qi]
    parent = torch.searchsorted(tb["steps"][1:].long(), qpos, right=True)
    qindex = qpos[torch.argsort(parent, stable=True)].int()
    counts = torch.bincount(parent, minlength=tb["neigh"].shape[0])
    steps_q = torch.cat([counts.new_zeros(1), torch.cumsum(counts, 0)]).int()
    ms = _event_ms(torch, lambda: fk.ops.selected_query_tables(
        xs, qindex, tb["steps"], steps_q, tb["neigh"], tb["cnt"], 32), flush)
    rows["selected_query_tables_room_k32"] = {
        "value": qi.numel() / (ms * 1e-3), "unit": "queries/s", "ms": ms,
        "what": "reference table ABI (FlashKNN_Selected_Query_DL boundary)"}
    # Morton keys and the 27 neighbour keys of the room's parent cells
    ms = _event_ms(torch, lambda: fk.ops.morton_encode(rgrid), flush)
    pgrid = torch.unique(rgrid >> 2, dim=0)
    nms = _event_ms(torch, lambda: fk.ops.morton_neighbor_keys(pgrid), flush)
    rows["morton_room"] = {"value": ms, "unit": "ms", "neighbor_keys_ms": nms,
                           "n_points": int(rgrid.shape[0]), "n_parents": int(pgrid.shape[0])}
    rows["self_query_cube_k16"] = row_cube(fk, torch, dev, flush)
    # LiDAR scan (C3), K=16, alpha 4 and alpha 8 (num_down 2 and 3)
    lo_ = torch.tensor([lx.shape[0]], device=dev)
    for nd, alpha in ((2, 4), (3, 8)):
        ms = _event_ms(torch, lambda: fk.ops.knn_offsets(lx, lo_, 16, synthetic.C3_VOXEL, nd),
                       flush)
        rows[f"self_query_lidar_k16_alpha{alpha}"] = {
            "value": lx.shape[0] / (ms * 1e-3), "unit": "queries/s", "ms": ms,
            "n_points": int(lx.shape[0])}
    # grouping: 16-cloud batch, K=16, 64 channels
    off = T(b.offsets)
    idx, _ = fk.ops.knn_offsets(bx, off, 16, synthetic.C4_VOXEL, 2)
    feat = torch.randn((len(b.xyz), 64), device=dev)
    ms = _event_ms(torch, lambda: fk.ops.group_features(feat, idx), flush)
    m, c = idx.numel(), 64
    algo = m * c * 4 + m * 4 + len(b.xyz) * c * 4
    rows["grouping_batch_c64_fwd"] = {
        "value": algo / (ms * 1e-3) / 1e9, "unit": "GB/s", "ms": ms,
        "roofline": {"bound": "hbm", "achieved": algo / (ms * 1e-3) / 1e9, "peak": peak_gbs,
                     "frac": algo / (ms * 1e-3) / 1e9 / peak_gbs,
                     "algorithmic_bytes": algo}}
    g = torch.randn((idx.shape[0], 16, 64), device=dev)
    gf = torch.empty_like(feat)
    ms = _event_ms(torch, lambda: fk.ops.group_backward(g, idx, len(b.xyz), 64, False, gf), flush)
    rows["grouping_batch_c64_bwd"] = {"value": ms, "unit": "ms"}
    return rows


def small_rows(args):
    """Only the small-problem rows (the uniform cube and the DeLA hierarchy):
    a short run for launch lists of those workloads."""
    import torch

    import flashknn_exprepo_b200 as fk
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    return {"rows": {"self_query_cube_k16": row_cube(fk, torch, dev, flush),
                     "hierarchy_lidar": row_hierarchy(fk, torch, dev)}}


def rows_only(args):
    """One distance backward on the 16-cloud batch and the per-path rows."""
    import torch

    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200 import synthetic
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    b = synthetic.uneven_batch()
    if args.clouds < len(b.counts):
        b = synthetic.first_clouds(b, args.clouds)
    x = torch.from_numpy(b.xyz).to(dev)
    off = torch.from_numpy(b.offsets).to(dev)
    idx, d = fk.ops.knn_offsets(x, off, args.k, synthetic.C4_VOXEL, 2)
    g = torch.from_numpy(synthetic.backward_weights(len(b.xyz), args.k)).to(dev)
    g = g * torch.isfinite(d).to(g.dtype)
    grad = torch.zeros_like(x)
    ms = _event_ms(torch, lambda: fk.ops.backward(x, x, idx, d, g, grad_q=grad, grad_p=grad,
                                                  accumulate=True), flush)
    return {"backward_ms": ms, "n_points": int(len(b.xyz)),
            "rows": rows_single_gpu(fk, torch, dev, flush, measured_peak_hbm()[0],
                                    clouds=args.clouds)}


def fd_check(fk, torch, dev, batch, k, voxel, count=2048, h=1e-4):
    """Max relative error (max-norm) of the backward's coordinate gradient of
    L = sum w * d against FP64 central finite differences (step h metres,
    neighbour indices held fixed) on a 2,048-point crop of the first cloud.
    A perturbed point changes only the terms of its own row and of the rows
    that name it, so only those are evaluated; the others cancel exactly."""
    from flashknn_exprepo_b200 import synthetic
    xyz = synthetic.crop(batch.xyz[: batch.offsets[0]], count,
                         np.random.default_rng(synthetic.SEED))
    n = len(xyz)
    x = torch.from_numpy(xyz).to(dev).requires_grad_(True)
    idx, d = fk.knn_query(k, x, torch.tensor([n], device=dev), voxel_size=voxel, num_down=2)
    w = synthetic.backward_weights(n, k)
    wt = torch.from_numpy(w).to(dev)
    (wt * torch.isfinite(d).to(wt.dtype) * d.nan_to_num(posinf=0.0)).sum().backward()
    got = x.grad.cpu().numpy().astype(np.float64)
    ii = np.where(np.isfinite(d.detach().cpu().numpy()), idx.cpu().numpy(), -1)
    w64 = w.astype(np.float64)
    x64 = xyz.astype(np.float64)
    rows_of = [[a] for a in range(n)]
    for r, t in zip(*np.nonzero(ii >= 0)):
        rows_of[ii[r, t]].append(r)

    def loss(xs, rows):
        sub = ii[rows]
        ok = sub >= 0
        dd = ((xs[rows][:, None, :] - xs[np.where(ok, sub, 0)]) ** 2).sum(-1)
        return float((np.where(ok, w64[rows], 0.0) * dd).sum())

    fd = np.zeros_like(x64)
    for a in range(n):
        rows = np.unique(rows_of[a])
        for c in range(3):
            xp = x64.copy()
            xm = x64.copy()
            xp[a, c] += h
            xm[a, c] -= h
            fd[a, c] = (loss(xp, rows) - loss(xm, rows)) / (2 * h)
    err = float(np.abs(got - fd).max() / max(np.abs(fd).max(), 1e-30))
    return {"max_rel_err": err, "target": 1e-4, "points": n, "h_m": h,
            "what": "FP64 central differences of sum(w * d), indices held fixed"}


def fp64_recall(batch, idx, k, per_cloud=256):
    """recall@K of the grid kNN against an exact FP64 brute force over whole
    clouds, on a seeded sample of queries per cloud; the brute force runs on
    every host core and is timed."""
    from oracle import oracle as O
    rng = np.random.default_rng(47)
    starts = np.concatenate([[0], batch.offsets[:-1]])
    rows = np.concatenate([np.sort(rng.choice(np.arange(s, e), min(per_cloud, e - s),
                                              replace=False))
                           for s, e in zip(starts, batch.offsets)])
    q_off = np.cumsum([min(per_cloud, e - s) for s, e in zip(starts, batch.offsets)])
    cores = cpu_cores()
    t0 = time.perf_counter()
    exact, _ = O.brute_knn_f64(batch.xyz, batch.offsets, k, batch.xyz[rows], q_off,
                               nthreads=cores)
    dt = time.perf_counter() - t0
    rec = O.set_recall(idx[rows], exact)
    return {"recall_at_k": float(rec.mean()), "rows": int(len(rows)),
            "fp64_brute_force": {"value": len(rows) / dt, "unit": "queries/s", "cores": cores,
                                 "sample": f"{per_cloud} seeded queries per cloud against "
                                           f"the whole cloud"}}


# ---------------------------------------------------------- reference arm

def run_reference(args):
    """The reference's CPU kNN path, timed on every host core: nanoflann
    (KD-tree, leaf 20, exact FP32 top-K, the reference's own nanoflann.hpp
    built into oracle/_ref) over every cloud of the batch, construction and
    query, one step = one pass over the 16 clouds.  Falls back to the oracle
    port of the grid path when the nanoflann build is missing.  Also reported:
    nanoflann on one thread (as the reference runs it), the oracle port, and
    the reference's own per-cloud GPU pipeline for context."""
    from flashknn_exprepo_b200 import synthetic
    from oracle import ref_nanoflann
    batch = synthetic.uneven_batch()
    k = args.k
    voxel = synthetic.C4_VOXEL
    cores = cpu_cores()
    n = int(len(batch.xyz))
    extra = {}
    if ref_nanoflann.available():
        cpu = nanoflann_rate(batch, k, max(1, args.steps), max(0, args.warmup))
        value = cpu["value"]
        sub = synthetic.first_clouds(batch, 2)
        _, _, tb, tq = ref_nanoflann.knn(sub.xyz, sub.offsets, k, nthreads=1)
        extra["nanoflann_single_thread"] = {
            "value": len(sub.xyz) / (tb + tq), "unit": "queries/s", "cores": 1,
            "sample": f"first 2 clouds ({len(sub.xyz)} points), build + query"}
        port = cpu_oracle_rate(batch.xyz, batch.offsets, k, voxel, budget_s=10.0)
        port.pop("seconds", None)
        extra["grid_port"] = port
    else:
        rates = []
        for _ in range(max(1, args.steps)):
            cpu = cpu_oracle_rate(batch.xyz, batch.offsets, k, voxel,
                                  budget_s=max(2.0, 60.0 / max(1, args.steps)))
            rates.append(cpu["value"])
        cpu.pop("seconds", None)
        value = statistics.median(rates)
        cpu["value"] = value
    line = {"impl": "reference", "metric": "kNN queries/s at K=16 (batched uneven 16-cloud, "
                                           "construction + query)",
            "value": value, "unit": "queries/s", "higher_is_better": True,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": n / value * 1e3,
            "dtype": "f32", "data": "synthetic (seeded, stands in for S3DIS/SemanticKITTI)",
            "config": {"workload": "uneven_batch_16clouds_k16", "n_points": n,
                       "k": k, "voxel_m": voxel, "num_down": 2},
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    line.update(extra)
    try:
        line["reference_gpu_per_cloud"] = reference_gpu_per_cloud(batch, k, voxel)
    except Exception as exc:  # context only: never fails the CPU arm
        line["reference_gpu_per_cloud"] = {"unavailable": f"{type(exc).__name__}: {exc}"[:200]}
    try:
        line["reference_kernel"] = reference_kernel_rows(batch)
    except Exception as exc:  # context only
        line["reference_kernel"] = {"unavailable": f"{type(exc).__name__}: {exc}"[:200]}
    return line


def reference_kernel_rows(batch):
    """The reference's production kernel alone (FlashKNN_Query_Dynamic_Load
    built for sm_100a) on the tables its own construction builds, timed with
    CUDA events around each call, L2 flushed before each: the room at K=32
    and the largest cloud of the uneven batch at K=16.  Our arm's rows
    query_tables_room_k32 / query_tables_largest_cloud_k16 time
    fknn_query_tables on the same tables (the tables are equal bit for bit:
    tests/test_gpu_reference_parity.py).  The reference launcher ends with a
    cudaDeviceSynchronize, so its closing event is recorded only after the
    host wakes up: `sync_gap_ms` is that gap measured alone (two events
    around a synchronise of an idle stream), an upper bound of what the
    events add to the kernel time."""
    import torch
    from flashknn_exprepo_b200 import synthetic
    from oracle import ref_kernels, ref_pipeline
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not ref_kernels.available():
        return {"unavailable": "reference kernels not built (oracle/build_ref.py)"}
    cufun = ref_kernels.load()
    dev = torch.device("cuda", 0)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    c = int(np.argmax(batch.counts))
    cases = [("room_k32", synthetic.room(), synthetic.C2_VOXEL, 32),
             ("largest_cloud_k16",
              batch.xyz[int(batch.offsets[c] - batch.counts[c]):int(batch.offsets[c])],
              synthetic.C4_VOXEL, 16)]
    out = {}
    for name, xyz, voxel, k in cases:
        x = torch.from_numpy(np.ascontiguousarray(xyz)).to(dev)
        grid = torch.floor(x * (1.0 / voxel)).long()
        t = ref_pipeline.reference_tables(cufun, grid, torch.zeros_like(grid[:, 0]), x, 2)
        ri = torch.zeros((len(xyz), k), dtype=torch.int32, device=dev)
        rd = torch.zeros((len(xyz), k), dtype=torch.float32, device=dev)
        ms = _event_ms(torch, lambda: cufun.FlashKNN_Query_Dynamic_Load(
            t["xyz_sorted"], t["steps"], t["neigh"], t["cnt"], k, ri, rd, 1, math.inf), flush)
        out[name] = {"value": len(xyz) / (ms * 1e-3), "unit": "queries/s", "ms": ms,
                     "n_points": int(len(xyz))}
    out["sync_gap_ms"] = _event_ms(torch, torch.cuda.synchronize, flush)
    return out


def reference_gpu_per_cloud(batch, k, voxel):
    import torch
    from oracle import ref_kernels, ref_pipeline
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not ref_kernels.available():
        return {"unavailable": "reference kernels not built (oracle/build_ref.py)"}
    cufun = ref_kernels.load()
    dev = torch.device("cuda", 0)
    starts = np.concatenate([[0], batch.offsets[:-1]])
    clouds = []
    for s, e in zip(starts, batch.offsets):
        x = torch.from_numpy(batch.xyz[s:e]).to(dev)
        g = torch.floor(x / voxel).long()
        clouds.append((g, torch.zeros(len(x), dtype=torch.long, device=dev), x))
    for g, b, x in clouds[:2]:
        ref_pipeline.reference_query(cufun, g, b, x, k)
    torch.cuda.synchronize()
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        for g, b, x in clouds:
            ref_pipeline.reference_query(cufun, g, b, x, k)
    dt = (time.perf_counter() - t0) / reps
    return {"value": len(batch.xyz) / dt, "unit": "queries/s", "ms_per_step": dt * 1e3,
            "what": "reference FlashKNN.query pipeline (ATen construction + "
                    "FlashKNN_Query_Dynamic_Load built for sm_100a), one call per cloud, "
                    "wall clock incl. its device synchronisations"}


# -------------------------------------------------------------------- main

def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args)))
        return

    if args.small_rows:
        print(json.dumps(small_rows(args)))
        return
    if args.rows_only:
        print(json.dumps(rows_only(args)))
        return

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        out = run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.barrier()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    k = args.k
    peak, peak_kind = measured_peak_hbm()
    kern = out["kernel_ms"]
    n_local = out["local_n"]
    algo_bytes = n_local * (12 + 8 * k) + 8 * n_local
    roofline = None
    if kern:
        avg = sum(kern) / len(kern)
        achieved = algo_bytes / (avg * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": profiled_traffic(k),
                    "kernel": f"fknn::k_query<{1 << max(0, (k - 1).bit_length())}>",
                    "kernel_ms": avg, "limiter": profiled_limiter(k),
                    "algorithmic_bytes_per_launch": algo_bytes,
                    "peak_source": f"{peak_kind} hbm_gbs"}
    line = {
        "metric": "kNN queries/s at K=16 (batched uneven 16-cloud, construction + query)",
        "value": out["value"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": out["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; stands in for S3DIS/SemanticKITTI crops)",
        "config": {"workload": f"uneven_batch_{args.clouds}clouds_k{k}", "n_points": out["n_points"],
                   "n_clouds": args.clouds * world, "k": k, "voxel_m": 0.05, "num_down": 2,
                   "step": "CUDA-graph replay of construction + query",
                   "l2": "flushed (256 MiB memset) before every timed step",
                   "parallelism": f"{world} x 16 clouds, whole clouds per GPU, no collective"},
        "e2e": out["e2e"], "gpu_launches": out["launches_per_step"] * args.steps,
        "clocks": out["clocks"], "roofline": roofline,
        "graph_matches_eager": out["graph_matches_eager"],
        "launch_shape": out["launch_shape"],
    }
    if "per_cloud" in out:
        line["per_cloud"] = out["per_cloud"]
        line["batched_vs_per_cloud"] = out["value"] / out["per_cloud"]["value"]
    if "per_cloud_graph" in out:
        line["per_cloud_graph"] = out["per_cloud_graph"]
        line["batched_vs_per_cloud_graph"] = out["value"] / out["per_cloud_graph"]["value"]
    if "batched_k32" in out:
        line["batched_k32"] = out["batched_k32"]
    if "fwd_bwd_ms" in out:
        line["fwd_bwd_ms"] = out["fwd_bwd_ms"]
    if "fd_check" in out:
        line["fd_check"] = out["fd_check"]
    if kern:
        line["phases_ms"] = {"construction": out["ms_per_step"] - roofline["kernel_ms"],
                             "query": roofline["kernel_ms"],
                             "backward": out.get("backward_ms")}
    if "recall" in out:
        line["recall"] = out["recall"]
    if "rows" in out:
        line["rows"] = out["rows"]
    if world == 1 and not args.no_extras:
        from flashknn_exprepo_b200 import synthetic
        b = synthetic.uneven_batch()
        from oracle import ref_nanoflann
        port = cpu_oracle_rate(b.xyz, b.offsets, k, synthetic.C4_VOXEL, budget_s=10.0)
        port.pop("seconds", None)
        if ref_nanoflann.available():
            line["cpu_baseline"] = nanoflann_rate(b, k, 3, 1)
            line["grid_port_cpu"] = port
        else:
            line["cpu_baseline"] = port
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
