#!/usr/bin/env python
"""Benchmark of the visibility-buffer rasterizer (one JSON line on rank 0).

A step is one frame of the plain path -- clear, stage 1/2/3, resolve to
RGBA8 -- of a seeded synthetic scene resident in HBM, timed with CUDA events
on the launching stream.  Metric: Gtris/s (triangles of the scene per second
of frame time).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                  [--impl ours|reference]

--impl reference runs the reference's own kernels (CuRast's
triangles_visbuffer.cu / resolve.cu built from its sources with its own
NVRTC recipe into oracle/_ref) on the same scene and GPU, through the
harness that launches them as CuRast's render host does.

With --gpus N > 1 (under torchrun) every rank renders its own replica of the
frame: the plain single-view path has no exchange step, so N GPUs are N
replicas and the value is the sum over ranks (weak scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "curast-ooc_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

L2_BYTES = 126 * 1024 * 1024


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def build_workload(name):
    """Seeded synthetic stand-ins for the reference's benchmark scenes.
    Host workloads hold numpy arrays, device workloads torch CUDA tensors."""
    import scenes

    if name == "heightfield_1m_1080p":
        W, H = 1920, 1080
        pos, idx, col = scenes.heightfield()
        view, proj = scenes.heightfield_camera(W, H)
        return dict(name=name, W=W, H=H, meshes=[(pos, idx, col)], instances=[(0, scenes.identity())],
                    view=view, proj=proj, device=False,
                    desc="1024x512-quad displaced heightfield (1,048,576 triangles, 525,825 vertices), 1920x1080")
    if name.startswith("instanced_"):
        # instanced_<K>x<N>m_1080p: one N-million-triangle mesh drawn as K instances
        k, n = name.split("_")[1].split("x")
        count, tris = int(k), int(n.rstrip("m")) * 1_000_000
        W, H = 1920, 1080
        pos, idx, col = scenes.asteroid(tris, device="cuda")
        view, proj = scenes.instanced_camera(W, H)
        return dict(name=name, W=W, H=H, meshes=[(pos, idx, col)],
                    instances=[(0, w) for w in scenes.instanced_field(count)], view=view, proj=proj, device=True,
                    desc=f"one seeded {tris:,}-triangle displaced icosphere drawn as {count} instances (uniform "
                         f"rotation, scale 0.5-2, positions uniform in a 100^3 box), 1920x1080")
    if name.startswith("planet_"):
        # planet_<N>m_1080p: the dense subdivided-sphere scene with N million triangles
        count = int(name.split("_")[1].rstrip("m")) * 1_000_000
        W, H = 1920, 1080
        pos, idx, col = scenes.planet(count, device="cuda", width=W, height=H)
        view, proj = scenes.planet_camera(W, H)
        return dict(name=name, W=W, H=H, meshes=[(pos, idx, col)], instances=[(0, scenes.identity())],
                    view=view, proj=proj, device=True,
                    desc=f"seeded displaced icosphere, {count:,} triangles, per-patch subdivision levels giving a "
                         f"lognormal pre-clip projected-area histogram, 1920x1080")
    raise SystemExit(f"unknown workload {name}")


def scene_counts(wl):
    def ntri(m):
        p, i, _ = wl["meshes"][m]
        return i.shape[0] if i is not None else p.shape[0] // 3

    T = sum(ntri(m) for m, _ in wl["instances"])
    V = sum(p.shape[0] for p, _, _ in wl["meshes"])
    Tunique = sum(ntri(m) for m in range(len(wl["meshes"])))
    return T, V, Tunique


def host_mesh(mesh):
    """numpy (positions, uint32 indices, uint32 colours) of a workload mesh."""
    p, i, c = mesh
    if hasattr(p, "cpu"):
        p = p.cpu().numpy()
        i = None if i is None else i.cpu().numpy().view(np.uint32)
        c = None if c is None else c.cpu().numpy().view(np.uint32)
    return p, i, c


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.out.name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
def init_dist(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def cpu_baseline(wl, budget_s=20.0):
    """The oracle (CPU restatement of the reference algorithm) on this host's
    cores, on a bounded sample of the same frame."""
    import oracle_lib as ol

    ncores = os.cpu_count() or 1
    pos, idx, col = host_mesh(wl["meshes"][0])
    T = idx.shape[0]
    sample = T
    t_used = 0.0
    while True:
        fr = ol.Frame([(pos, idx[:sample], col, wl["instances"][0][1])], wl["view"])
        t0 = time.perf_counter()
        ol.raster(fr, wl["W"], wl["H"], wl["proj"][5], nthreads=ncores)
        dt = time.perf_counter() - t0
        t_used += dt
        if sample == T or t_used > budget_s / 2 or dt > budget_s / 4:
            break
        sample = min(T, int(sample * 4))
    return {"value": sample / dt / 1e9, "unit": "Gtris/s", "cores": ncores, "kind": "port",
            "sample": f"oracle raster of triangles [0, {sample}) of the same frame ({sample / T:.0%}), "
                      f"all {ncores} host threads (OpenMP), {dt:.2f} s"}


def read_traffic(kernel, workload):
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1]))
    except OSError:
        pass
    return None


def run_ours(args, rank, world, local):
    import torch

    import pycurast as pc

    wl = build_workload(args.workload)
    T, V, Tu = scene_counts(wl)
    W, H = wl["W"], wl["H"]
    ctx = pc.Context(device=local)
    if wl["device"]:
        handles = [ctx.mesh_from_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
                   for (p, i, c) in wl["meshes"]]
    else:
        handles = [ctx.mesh_from_host(p, i, c) for (p, i, c) in wl["meshes"]]
    inst = pc.make_instances([(handles[m], w) for m, w in wl["instances"]])
    cam = pc.make_camera(wl["view"], wl["proj"], W, H)
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    host_rgba = torch.empty(W * H, dtype=torch.int32, pin_memory=True)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    geom_bytes = 12 * Tu + 12 * V
    flush = None
    if geom_bytes + 12 * W * H < 2 * L2_BYTES:
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")

    # warm-up (the first frame sizes the queues)
    ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_SYNC, stream=sh)
    for _ in range(max(args.warmup - 1, 0)):
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=0, stream=sh)
    ctx.sync()
    st, fstats = ctx.stats()
    ctx.drain_stage_times()

    # ---- device-timed region: inputs resident in HBM --------------------
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        if flush is not None:
            flush.fill_(k)
        evs[k][0].record(stream)
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_TIMING, stream=sh)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop() if clocks else None
    ctx.sync()
    ms_steps = [a.elapsed_time(b) for a, b in evs]
    ms = max_over_ranks(float(np.mean(ms_steps)), world)
    stage_ms, nframes = ctx.drain_stage_times()
    stage_ms = {k: v / max(nframes, 1) for k, v in stage_ms.items()}

    # ---- end to end: host instance list + camera in, RGBA8 image out ------
    barrier(world)
    torch.cuda.synchronize()
    e2e_ms = []
    for k in range(args.steps):
        if flush is not None:
            flush.fill_(k)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=0, stream=sh)
        host_rgba.copy_(rgba, non_blocking=True)
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    ctx.sync()
    e2e = max_over_ranks(float(np.mean(e2e_ms)), world)
    n = len(wl["instances"])
    h2d = 3 * ((n * 64 + 255) // 256 * 256) + (48 + 255) // 256 * 256

    if rank != 0:
        return None
    peak, peak_kind = load_peaks()
    # Algorithmic bytes per launch.  vertex pass: 12 B position read + 1 B
    # outcode write per (instance, vertex); stage 1: 12 B index tile per
    # triangle + each outcode byte once; whole frame: the reference's
    # 12T + 12V + 16P (index and vertex fetch once, visbuffer clear + write)
    # plus the resolve's 12P.
    nV_inst = sum(wl["meshes"][m][0].shape[0] for m, _ in wl["instances"])
    algo = {"vertex": 13 * nV_inst, "stage1": 12 * T + nV_inst}
    dominant = max(("vertex", "stage1", "stage2", "stage3", "resolve", "clear"), key=lambda s: stage_ms[s])
    rk = "stage1" if dominant not in algo else dominant
    t_k = stage_ms[rk]
    achieved = algo[rk] / (t_k * 1e-3) / 1e9
    frame_bytes = 12 * T + 12 * V + 16 * W * H + 12 * W * H
    frame_gbs = frame_bytes / (ms * 1e-3) / 1e9
    line = {
        "metric": "Gtris/s @1080p (plain 3-stage visbuffer + resolve, one frame per step)",
        "value": world * T / (ms * 1e-3) / 1e9,
        "unit": "Gtris/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "triangles": T, "vertices": V,
                   "width": W, "height": H, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps" if flush is not None else "inputs larger than L2",
                   "stage_ms": stage_ms, "dominant_stage": dominant,
                   "nontrivial": int(fstats.nontrivial), "huge_tiles": int(fstats.huge_tiles),
                   "frame_roofline": {"bytes": frame_bytes, "achieved_gbs": frame_gbs,
                                      "frac": frame_gbs / peak}},
        "e2e": {"value": world * T / (e2e * 1e-3) / 1e9, "unit": "Gtris/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4 * W * H},
        "roofline": {"kernel": f"k_{rk}", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": algo[rk], "kernel_ms": t_k,
                     "traffic": read_traffic(rk, wl["name"])},
        "gpu_launches": 6 * args.steps,
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl)
    ctx.close()
    return line


# ---------------------------------------------------------------------------
# the reference's own kernels
# ---------------------------------------------------------------------------
def run_reference(args, rank, world, local):
    if rank != 0:
        return None
    import oracle_lib as ol

    wl = build_workload(args.workload)
    T, V, Tu = scene_counts(wl)
    W, H = wl["W"], wl["H"]
    try:
        ref = ol.Reference("native", device=local)
    except Exception as e:  # noqa: BLE001
        return {"impl": "reference", "unavailable": f"reference kernels not loadable: {e}"}
    if wl["device"]:
        ids = [ref.mesh_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
               for (p, i, c) in wl["meshes"]]
    else:
        ids = [ref.mesh_host(p, i, c) for (p, i, c) in wl["meshes"]]
    mids = [ids[m] for m, _ in wl["instances"]]
    worlds = np.stack([np.asarray(w, np.float32).reshape(16) for _, w in wl["instances"]])
    # The reference never checks its queue capacities: size them from the CPU
    # oracle's exact counts for this frame, with a wide margin (the fast-math
    # build decides a handful of edge triangles differently).
    items = []
    for m, w in wl["instances"]:
        p, i, c = host_mesh(wl["meshes"][m])
        items.append((p, i, c, w))
    _, ost = ol.raster(ol.Frame(items, wl["view"]), W, H, wl["proj"][5], nthreads=os.cpu_count() or 1)
    del items
    cap_nt = min(T, 2 * int(ost.nontrivial) + (1 << 20))
    cap_huge = 2 * int(ost.huge_tiles) + (1 << 20)
    ref.frame(mids, worlds, wl["view"], wl["proj"], W, H, instanced=True, cap_nontrivial=cap_nt,
              cap_huge=cap_huge, frames=max(args.warmup, 1), want_color=False)
    _, _, _, ms, counts = ref.frame(mids, worlds, wl["view"], wl["proj"], W, H, instanced=True,
                                    cap_nontrivial=cap_nt, cap_huge=cap_huge, frames=args.steps, want_color=False)
    step_ms = float(ms[0] + ms[1])
    v = T / (step_ms * 1e-3) / 1e9
    return {
        "impl": "reference",
        "metric": "Gtris/s @1080p (plain 3-stage visbuffer + resolve, one frame per step)",
        "value": v,
        "unit": "Gtris/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "triangles": T, "vertices": V, "width": W,
                   "height": H, "parallelism": "single GPU", "stage_ms": {"clear+raster": float(ms[0]),
                                                                          "resolve": float(ms[1])},
                   "nontrivial": int(counts[0]), "huge_tiles": int(counts[1]),
                   "build": "CuRast NVRTC recipe (--use_fast_math, LTO) for sm_100a"},
        "cpu_baseline": {"kind": "reference", "value": v, "unit": "Gtris/s", "cores": 0,
                         "sample": "not a CPU run: the reference has no CPU rasterizer, so its own CUDA kernels "
                                   "are timed on this B200 (whole frame)"},
        "e2e": {"value": v, "unit": "Gtris/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="planet_400m_1080p",
                    help="planet_400m_1080p (the 400M-triangle dense mesh), planet_<N>m_1080p, heightfield_1m_1080p")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    rank, world, local = init_dist(args)
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world, local)
        else:
            line = run_ours(args, rank, world, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
