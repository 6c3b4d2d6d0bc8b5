"""Benchmark of the batched nearest-hit query path on one or more B200s.

Workload (one "step"): nearest-hit raycast of 1,048,576 rays -- half coherent
(a 1024 x 512 camera grid at z = 200, within 2 degrees of -z), half
incoherent (uniform origins in the scene box, isotropic directions) --
against a 1,048,576-triangle height field (1024 x 512 cells, 6 random-phase
sinusoids of amplitude 1-20 plus N(0, 0.5) noise), t_max 2000; seeded
synthetic data (the reference publishes no dataset).

Metric: Mrays/s. ``value`` is device-timed throughput with rays resident in
HBM (CUDA events around each launch on the launching stream, L2 flushed by a
256 MiB write between steps, outside the timed events); ``e2e`` is the same
metric through the host-buffer C ABI call (pinned host rays in, leaf / toi /
normal out, copies inside the timed region). Multi-GPU runs are weak-scaled:
every rank answers its own 1,048,576-ray batch against its own replica of
the scene, with no collective on the data path; time is the max over ranks.

``--impl reference`` times the reference's CPU algorithm (the oracle's C++
restatement of Bvh::raycast_nearest_batch_parallel, all host threads) on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s nearest-hit, 1M tris; learned-seeded vs plain GPU, identical hits"
WORKLOAD = ("terrain height field 1024x512 cells = 1,048,576 triangles; 1,048,576 rays per step "
            "(524,288 coherent + 524,288 incoherent); raycast_nearest, t_max 2000, default filter")
RAY_BYTES = 24    # origin[3], dir[3] f32
OUT_BYTES = 20    # leaf u32, toi f32, normal[3] f32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--order", default="near_first", choices=["near_first", "reference"])
    ap.add_argument("--rays", type=int, default=1 << 20,
                    help="rays per step (half coherent, half incoherent); the metric is quoted at 1,048,576")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the traversal kernel from the committed ncu
    summary (profiles/ray_nearest_terrain.md), or None."""
    p = os.path.join(ROOT, "profiles", "ray_nearest_terrain.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("traffic_bytes_per_launch"):
            try:
                return int(line.split("=")[1].strip().split()[0].replace(",", ""))
            except (IndexError, ValueError):
                return None
    return None


def cpu_baseline_sample(s, threads: int):
    """The oracle (C++ restatement of the reference CPU batch) on the host."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    sc = O.Scene("tris", 3, s["prims"])
    build_s = time.perf_counter() - t0
    rays = s["rays"]
    n = rays.shape[0]
    sc.nearest(rays[:4096], s["max_toi"], threads=threads)  # warm
    t0 = time.perf_counter()
    sc.nearest(rays, s["max_toi"], threads=threads)
    dt = time.perf_counter() - t0
    return dict(value=n / dt / 1e6, unit="Mrays/s", cores=threads, kind="port",
                sample=f"all {n} rays of the workload, one pass, {threads} threads, contiguous chunks "
                       f"(Bvh::raycast_nearest_batch_parallel semantics); tree build {build_s:.2f} s not counted")


def run_reference(args, rank, world):
    if rank != 0:
        return
    from spatial_query_b200 import scenes
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    s = scenes.terrain_scene(seed=1)
    threads = os.cpu_count() or 1
    sc = O.Scene("tris", 3, s["prims"])
    per_step = 131072
    rays = s["rays"]
    n = rays.shape[0]
    # Each step is a bounded sample: 131,072 rays, half from each ray kind.
    def sample(i):
        h = per_step // 2
        a = (i * h) % (n // 2)
        return np.concatenate([rays[a:a + h], rays[n // 2 + a:n // 2 + a + h]])
    for i in range(args.warmup):
        sc.nearest(sample(i), s["max_toi"], threads=threads)
    times = []
    for i in range(args.steps):
        q = sample(args.warmup + i)
        t0 = time.perf_counter()
        sc.nearest(q, s["max_toi"], threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1000 * sum(times) / len(times)
    v = per_step / (ms / 1000) / 1e6
    line = {"metric": METRIC, "value": round(v, 3), "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "sample_rays_per_step": per_step},
            "cpu_baseline": {"value": round(v, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"{per_step} rays per step (half coherent, half incoherent), oracle C++ "
                                       f"restatement of Bvh::raycast_nearest_batch_parallel, {threads} threads"},
            "e2e": {"value": round(v, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import spatial_query_b200 as sq
    from spatial_query_b200 import scenes

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    s = scenes.terrain_scene(seed=1)
    if rank > 0:
        # Weak scaling: each rank its own ray batch of the same two kinds.
        s2 = scenes.terrain_scene(seed=1 + 1000 * rank)
        s["rays"] = s2["rays"]
    if args.rays != s["rays"].shape[0]:
        half, total = args.rays // 2, s["rays"].shape[0]
        s["rays"] = np.ascontiguousarray(np.concatenate([s["rays"][:half], s["rays"][total // 2: total // 2 + half]]))
    n = s["rays"].shape[0]
    geom = sq.Geometry("tris", 3, s["prims"])
    tree = sq.HostBvh.build(geom)
    ctx = sq.Context(local)
    # Every kernel, flush and event goes on the context's own stream.
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    torch.cuda.set_stream(stream)
    ctx.set_order(sq.ORDER_REFERENCE if args.order == "reference" else sq.ORDER_NEAR_FIRST)
    scene = sq.DeviceBvh(ctx, tree, geom)
    info = scene.info()

    dev = torch.device("cuda", local)
    d_rays = torch.from_numpy(s["rays"]).to(dev)
    d_leaf = torch.empty(n, dtype=torch.int32, device=dev)
    d_toi = torch.empty(n, dtype=torch.float32, device=dev)
    d_nrm = torch.empty((n, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        scene.raycast_nearest_d(d_rays, n, s["max_toi"], d_leaf, d_toi, d_nrm)

    # Instrumented run (untimed): per-batch counters for the algorithmic bytes.
    st = scene.raycast_nearest_d(d_rays, n, s["max_toi"], d_leaf, d_toi, d_nrm, stats=True)
    torch.cuda.synchronize()
    replayed = ctx.last_replay_count if args.order == "near_first" else 0
    fetches = (st["nodes_visited"] - n) // 2          # child-pair records read
    alg_bytes = (fetches * info["node_record_bytes"] + st["narrow_tests"] * info["prim_record_bytes"]
                 + n * (RAY_BYTES + OUT_BYTES))

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = ctx.launch_count
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    launches = ctx.launch_count - launches0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms = sum(step_ms) / len(step_ms)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1000) / 1e6

    # End to end through the host-buffer C ABI: pinned rays in, hits out.
    h_rays = torch.from_numpy(s["rays"]).pin_memory()
    h_leaf = torch.empty(n, dtype=torch.int32).pin_memory()
    h_toi = torch.empty(n, dtype=torch.float32).pin_memory()
    h_nrm = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    import ctypes as C
    hits = sq._Hits(h_leaf.data_ptr(), h_toi.data_ptr(), None, h_nrm.data_ptr(), None)

    def e2e_step():
        ctx.check(sq.lib().sq_raycast_nearest(ctx.h, scene.h, h_rays.data_ptr(), n, s["max_toi"], None, None,
                                              C.byref(hits), None), "sq_raycast_nearest")

    for _ in range(max(2, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    e_ms = []
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        b.synchronize()
        e_ms.append(a.elapsed_time(b))
    e2e_ms = sum(e_ms) / len(e_ms)
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * n / (e2e_ms / 1000) / 1e6
    # The e2e results equal the device-resident results.
    assert torch.equal(h_leaf, d_leaf.cpu()) and torch.equal(h_toi.view(torch.int32), d_toi.cpu().view(torch.int32))

    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms / 1000) / 1e9
    traffic = profiled_traffic()
    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline_sample(s, os.cpu_count() or 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded height field and rays)",
            "config": {"workload": WORKLOAD, "path": f"plain GPU traversal, {args.order} order",
                       "replayed_in_reference_order": int(replayed),
                       "l2": "flushed between steps (256 MiB write, outside the timed events)",
                       "parallelism": f"replicated scene, rays sharded per rank (dp{world})",
                       "tree": {"nodes": info["n_nodes"], "depth": info["max_depth"],
                                "node_record_bytes": info["node_record_bytes"],
                                "prim_record_bytes": info["prim_record_bytes"]}},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                         "alg_bytes_per_launch": int(alg_bytes),
                         "alg_bytes_per_ray": round(alg_bytes / n, 1),
                         "counts_per_ray": {"node_records": round(fetches / n, 2),
                                            "narrow_tests": round(st["narrow_tests"] / n, 2)}},
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": n * RAY_BYTES,
                    "d2h_bytes_per_step": n * OUT_BYTES, "ms_per_step": round(e2e_ms, 4)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    scene.close()
    ctx.close()


if __name__ == "__main__":
    main()
