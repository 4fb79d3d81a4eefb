#!/usr/bin/env python
"""Benchmark of the visibility-buffer rasterizer (one JSON line on rank 0).

A step is one frame of the plain path -- clear, stage 1/2/3, resolve to
RGBA8 -- of a seeded synthetic scene resident in HBM, timed with CUDA events
on the launching stream.  Metric: Gtris/s (triangles of the scene per second
of frame time).  e2e is the same metric through the C ABI with every step's
frame table uploaded from page-locked memory and its RGBA8 image read back to
page-locked memory: steps back to back, each image copied on a second stream
while the next step renders into the other of two image buffers, timed from
the first step's start to the last image's arrival (the one-step-at-a-time
latency is reported beside it).

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
    Host workloads hold numpy arrays, device workloads torch CUDA tensors.
    A "_c" suffix renders the same scene's meshes in the reference's
    compressed format (bit-packed indices, 16-bit positions)."""
    import scenes

    if name.endswith("_c"):
        import pycurast as pc

        import oracle_lib as ol

        wl = build_workload(name[:-2])
        comps, decoded = [], []
        for mesh in wl["meshes"]:
            p, i, c = host_mesh(mesh)
            comp = pc.compress_mesh(p, i)
            comps.append(comp)
            dp, di = ol.decode_compressed(comp.packed, i.size, comp.index_min, comp.index_max, comp.positions,
                                          comp.aabb_min, comp.aabb_max)
            decoded.append((dp, di, c))
        wl.update(name=name, compressed=comps, decoded=decoded,
                  desc=wl["desc"] + "; meshes in the reference's compressed format (IX_PU16: bit-packed indices, "
                                    "16-bit quantised positions)")
        return wl

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
        # planet_<N>m_1080p: the dense subdivided-sphere scene with N million
        # triangles, camera just above the surface; planet_orbit_<N>m_1080p:
        # the same mesh seen whole from outside (its geometry must be read)
        parts = name.split("_")
        orbit = parts[1] == "orbit"
        count = int(parts[2 if orbit else 1].rstrip("m")) * 1_000_000
        W, H = 1920, 1080
        pos, idx, col = scenes.planet(count, device="cuda", width=W, height=H)
        view, proj = scenes.planet_orbit_camera(W, H) if orbit else scenes.planet_camera(W, H)
        where = ("seen whole from 2.6 radii (about half of the triangles face the camera, all of them in the frustum)"
                 if orbit else "camera 0.035 radii above the surface")
        return dict(name=name, W=W, H=H, meshes=[(pos, idx, col)], instances=[(0, scenes.identity())],
                    view=view, proj=proj, device=True,
                    desc=f"seeded displaced icosphere, {count:,} triangles, per-patch subdivision levels giving a "
                         f"lognormal pre-clip projected-area histogram, {where}, 1920x1080")
    if name.startswith("batched_"):
        # batched_<V>v_<N>m: N-million-triangle terrain seen by V seeded cameras
        nv_s, n_s = name.split("_")[1:3]
        nv = int(nv_s.rstrip("v"))
        tris = int(n_s.rstrip("m")) * 1_000_000
        quads = int(round((tris / 2) ** 0.5))
        pos, idx, col = scenes.terrain(n=quads, device="cuda")
        cams = scenes.batch_cameras(nv)
        return dict(name=name, meshes=[(pos, idx, col)], instances=[(0, scenes.identity())], cams=cams,
                    device=True, batched=True,
                    desc=f"seeded fractal-displaced grid of {quads}x{quads} quads ({idx.shape[0]:,} triangles) seen "
                         f"by {nv} seeded cameras, resolutions uniform among 512x512, 1280x720, 1920x1080, "
                         f"3840x2160")
    if name.startswith("post_"):
        # post_2160p_ss2: EDL + SSAO + the 2x supersampled display resolve of a
        # 3840x2160 colorbuffer (the 1M-triangle heightfield) to 1920x1080
        W, H, oW, oH = 3840, 2160, 1920, 1080
        pos, idx, col = scenes.heightfield()
        view, proj = scenes.heightfield_camera(W, H)
        return dict(name=name, W=W, H=H, outW=oW, outH=oH, meshes=[(pos, idx, col)],
                    instances=[(0, scenes.identity())], view=view, proj=proj, device=False, post=True,
                    desc="eye-dome lighting + ambient occlusion (32 samples, 7x7 blur) + 2x2 supersampled display "
                         "resolve of the 3840x2160 colorbuffer of the 1M-triangle heightfield, to 1920x1080")
    if name.startswith("glb_"):
        # glb_<N>m: a binary glTF file of N one-million-triangle primitives
        # (u32 indices, RGBA8 colours, one node each), in host memory
        n = int(name.split("_")[1].rstrip("m"))
        return dict(name=name, glb=True, primitives=n,
                    desc=f"binary glTF file of {n} primitives of 1,048,576 triangles (1024x512-quad heightfield "
                         f"patches: float VEC3 positions, u32 indices, VEC4 u8 colours), one node with a matrix "
                         f"each, read from host memory into resident meshes and an instance list")
    if name.startswith("served_"):
        # served_<R>rps: Poisson requests at R/s over three resident scenes,
        # beside a 4e9-triangle out-of-core scene streamed from pinned host
        # memory
        return dict(name=name, rate=float(name.split("_")[1].rstrip("rps")), served=True, device=True,
                    desc="Poisson-arriving requests over three resident scenes (1M-triangle heightfield, 60M-triangle "
                         "terrain, 400M-triangle planet), resolutions uniform among 512x512, 1280x720, 1920x1080, "
                         "3840x2160, under a 64 GiB framebuffer/queue budget; beside them a 3.997e9-triangle terrain "
                         "of 61,009 nodes (<= 65,536 triangles each) in 72 GB of pinned host memory streamed under "
                         "a 32 GiB geometry budget")
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
def step_spread(ms_steps):
    """Median and 99th percentile of the per-step times (this rank)."""
    a = np.asarray(ms_steps, np.float64)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "steps": int(a.size)}


def init_dist(args, backend=None):
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the
    launcher).  NCCL on GPUs; gloo when there is no GPU (the CPU tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = backend or ("nccl" if cuda else "gloo")
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    """The slowest rank's time: every multi-GPU number is max over ranks."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, ms_max, world):
    """Whole-job throughput of N replicas: every rank processed units_per_rank
    in at most ms_max (weak scaling)."""
    return world * units_per_rank / (ms_max * 1e-3)


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


def frame_parity(wl, ctx, inst, vis, rgba, nthreads=None):
    """The bench's last frame against the CPU oracle's rendering of the same
    frame (instances in the order cr_render draws them): visbuffer bit for
    bit, RGBA8 within 1 per 8-bit channel.  Returns the parity record and the
    oracle's raster time of the whole frame (seconds)."""
    import oracle_lib as ol

    nthreads = nthreads or os.cpu_count() or 1
    W, H = wl["W"], wl["H"]
    order, _, _ = ctx.frame_assemble(inst, wl["view"])
    meshes = wl["decoded"] if wl.get("compressed") else [host_mesh(m) for m in wl["meshes"]]
    items = [(*meshes[wl["instances"][k][0]], wl["instances"][k][1]) for k in order]
    fr = ol.Frame(items, wl["view"])
    t0 = time.perf_counter()
    fb, ost = ol.raster(fr, W, H, wl["proj"][5], nthreads=nthreads)
    dt = time.perf_counter() - t0
    _, orgba = ol.resolve(fr, wl["view"], wl["proj"], W, H, fb, nthreads=nthreads)
    got = vis.cpu().numpy().view(np.uint64)
    img = rgba.cpu().numpy().view(np.uint32)
    bad = int((got != fb).sum())
    ch = int(np.abs(img.view(np.uint8).astype(np.int16) - orgba.view(np.uint8).astype(np.int16)).max())
    rec = {"visbuffer": "bit-exact" if bad == 0 else f"{bad} of {W * H} pixels differ",
           "rgba_max_channel_diff": ch, "pixels": W * H, "covered": int((fb != np.uint64(0xFFFFFFF000000000)).sum()),
           "oracle_nontrivial": int(ost.nontrivial), "oracle_huge_tiles": int(ost.huge_tiles),
           "checked": "the last timed frame against the CPU oracle (IEEE restatement of the reference kernels)"}
    del fr, items, meshes
    return rec, dt, bad == 0 and ch <= 1


def read_traffic(kernel, workload):
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1]))
    except OSError:
        pass
    return None


def plain_algorithmic_bytes(wl, fstats, T):
    """Algorithmic bytes per launch of the plain frame's kernels, from the
    units the frame processed (its stats).  The frame cull (timed with the
    vertex pass) reads a 24-byte box per vertex chunk and per work item and
    writes 8 B per listed item; the slice stamps read each listed item's
    entry and slice windows (8 + 32 B) and write a few 4-byte stamps (16 B
    counted); the vertex pass reads 12 B of position and writes one record
    (4-byte cell records up to 4096 pixels a side, else 8) per vertex of each
    slice it evaluates (the 128-vertex slices of the chunks its box did not
    classify that hold a vertex of a drawn item); stage 1 reads the
    12-byte index triple of every triangle of each drawn work item, the
    record of each vertex those triangles use once (counted as one per two
    triangles, as in a closed mesh, and at most the records written), and
    writes and reads 8 B per survivor of the records.
    Frames that draw a mesh more than once cull from box proofs and per-item
    vertex lists (no per-vertex records in device memory).  Returns (bytes per
    stage, triangles in drawn items, vertices evaluated)."""
    mids = [m for m, _ in wl["instances"]]
    direct = len(set(mids)) < len(mids)
    rec = 4 if max(wl["W"], wl["H"]) <= 4096 else 8
    items, items_drawn = int(fstats.work_items), int(fstats.work_items_drawn)
    chunks, chunks_eval = int(fstats.vertex_chunks), int(fstats.vertex_chunks_evaluated)
    slices_eval = int(getattr(fstats, "vertex_slices_evaluated", 0))
    surv = int(getattr(fstats, "stage1_survivors", 0))
    nV_inst = sum(wl["meshes"][m][0].shape[0] for m, _ in wl["instances"])
    stamps = 56 * items_drawn if slices_eval else 0
    if direct:
        # frame cull: one 24-byte item box per item (the instance matrices
        # stay in L1) and 8 B per listed item; stage 1: the 1408-byte vertex
        # list block of each listed item and the positions of its distinct
        # vertices (at most 128 x 12 B for these meshes)
        v_eval, tri_drawn = 0, min(T, items_drawn * 128)
        algo = {"vertex": 24 * items + 8 * items_drawn,
                "stage1": (1408 + 12 * 128) * items_drawn, "boxes": True}
    elif chunks:
        # the vertex pass evaluates the slices (128 vertices) of its listed
        # chunks that hold a vertex of a drawn item
        v_eval = min(nV_inst, slices_eval * 128 if slices_eval else chunks_eval * 1024)
        tri_drawn = min(T, items_drawn * 128)
        algo = {"vertex": 24 * (chunks + items) + (12 + rec) * v_eval + 8 * items_drawn + stamps,
                "stage1": 12 * tri_drawn + rec * min(v_eval, tri_drawn // 2) + 16 * surv}
    else:
        v_eval, tri_drawn = nV_inst, T
        algo = {"vertex": (12 + rec) * nV_inst, "stage1": 12 * T + rec * min(nV_inst, T // 2) + 16 * surv}
    if wl.get("compressed"):
        # compressed meshes: 6-byte positions, 3 x bits / 8 bytes of indices per triangle
        ib = 3 * wl["compressed"][0].bits / 8.0
        algo = {"vertex": 24 * (chunks + items) + (6 + rec) * v_eval + 8 * items_drawn + stamps,
                "stage1": ib * tri_drawn + rec * min(v_eval, tri_drawn // 2) + 16 * surv}
    return algo, tri_drawn, v_eval


def run_ours(args, rank, world, local):
    import torch

    import pycurast as pc

    wl = build_workload(args.workload)
    if wl.get("batched"):
        return run_batched(args, rank, world, local, wl)
    if wl.get("served"):
        return run_served(args, rank, world, local, wl)
    if wl.get("post"):
        return run_post(args, rank, world, local, wl)
    if wl.get("glb"):
        return run_glb(args, rank, world, local, wl)
    T, V, Tu = scene_counts(wl)
    W, H = wl["W"], wl["H"]
    ctx = pc.Context(device=local)
    if wl.get("compressed"):
        handles = [ctx.mesh_compressed(comp, dec[2]) for comp, dec in zip(wl["compressed"], wl["decoded"])]
    elif wl["device"]:
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
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=0, stream=sh)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop() if clocks else None
    ctx.sync()
    ms_steps = [a.elapsed_time(b) for a, b in evs]
    ms = max_over_ranks(float(np.mean(ms_steps)), world)
    # per-stage times from as many frames again, with events between the
    # stages (they keep consecutive kernels from overlapping, so the frame
    # times above are taken without them)
    ctx.drain_stage_times()
    for k in range(args.steps):
        if flush is not None:
            flush.fill_(k)
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_TIMING, stream=sh)
    torch.cuda.synchronize()
    ctx.sync()
    stage_ms, nframes = ctx.drain_stage_times()
    stage_ms = {k: v / max(nframes, 1) for k, v in stage_ms.items()}

    # ---- end to end: host instance list + camera in, RGBA8 image out ------
    # One step at a time (latency): the frame table goes up from page-locked
    # staging inside cr_render, the image comes back to page-locked memory.
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
    e2e_latency = max_over_ranks(float(np.mean(e2e_ms)), world)
    # Steps back to back (throughput), as a renderer streams frames: each
    # step's image is read back on a copy stream while the next step renders
    # into the other of two RGBA8 buffers; timed from the first step's start
    # to the last image's arrival in host memory.
    copy_stream = torch.cuda.Stream(device=local)
    rgba_b = [rgba, torch.empty_like(rgba)]
    host_b = [host_rgba, torch.empty(W * H, dtype=torch.int32, pin_memory=True)]
    rendered = [torch.cuda.Event(), torch.cuda.Event()]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    barrier(world)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(args.steps):
        j = k % 2
        if flush is not None:
            flush.fill_(k)
        if k >= 2:
            stream.wait_event(copied[j])  # step k-2's image has left this buffer
        ctx.render(inst, cam, vis.data_ptr(), rgba_b[j].data_ptr(), flags=0, stream=sh)
        rendered[j].record(stream)
        copy_stream.wait_event(rendered[j])
        with torch.cuda.stream(copy_stream):
            host_b[j].copy_(rgba_b[j], non_blocking=True)
        copied[j].record(copy_stream)
    for j in range(min(2, args.steps)):
        stream.wait_event(copied[j])
    b.record(stream)
    b.synchronize()
    ctx.sync()
    e2e = max_over_ranks(a.elapsed_time(b) / args.steps, world)
    # the last image arrived whole
    last = (args.steps - 1) % 2
    assert np.array_equal(host_b[last].numpy(), rgba_b[last].cpu().numpy())
    n = len(wl["instances"])
    h2d = 3 * ((n * 64 + 255) // 256 * 256) + (48 + 255) // 256 * 256

    if rank != 0:
        ctx.close()
        return None
    parity, oracle_s, parity_ok = (None, None, None)
    if not args.no_parity:
        parity, oracle_s, parity_ok = frame_parity(wl, ctx, inst, vis, rgba)
    peak, peak_kind = load_peaks()
    algo, tri_drawn, v_eval = plain_algorithmic_bytes(wl, fstats, T)
    items, items_drawn = int(fstats.work_items), int(fstats.work_items_drawn)
    chunks, chunks_eval = int(fstats.vertex_chunks), int(fstats.vertex_chunks_evaluated)
    dominant = max(("vertex", "stage1", "stage2", "stage3", "resolve", "clear"), key=lambda s: stage_ms[s])
    rk = "stage1" if dominant not in algo else dominant
    t_k = stage_ms[rk]
    achieved = algo[rk] / (t_k * 1e-3) / 1e9
    frame_bytes = 12 * T + 12 * V + 16 * W * H + 12 * W * H
    if wl.get("compressed"):
        frame_bytes = int(3 * wl["compressed"][0].bits / 8.0 * T) + 6 * V + 16 * W * H + 12 * W * H
    frame_gbs = frame_bytes / (ms * 1e-3) / 1e9
    line = {
        "metric": "Gtris/s @1080p (plain 3-stage visbuffer + resolve, one frame per step)",
        "value": replica_throughput(T, ms, world) / 1e9,
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
                   "stage_ms": stage_ms, "dominant_stage": dominant, "step_ms": step_spread(ms_steps),
                   "nontrivial": int(fstats.nontrivial), "huge_tiles": int(fstats.huge_tiles),
                   "hierarchical_cull": {"work_items": items, "work_items_drawn": items_drawn,
                                         "vertex_chunks": chunks, "vertex_chunks_evaluated": chunks_eval,
                                         "vertex_slices_evaluated": int(getattr(fstats, "vertex_slices_evaluated", 0)),
                                         "triangles_in_drawn_items": tri_drawn,
                                         "stage1_survivors": int(fstats.stage1_survivors)},
                   "frame_roofline": {"bytes": frame_bytes, "achieved_gbs": frame_gbs,
                                      "frac": frame_gbs / peak,
                                      "note": "reference formula 12T+12V+28P; provably culled groups are not "
                                              "read, so this can exceed 1"}},
        "e2e": {"value": world * T / (e2e * 1e-3) / 1e9, "unit": "Gtris/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4 * W * H,
                "mode": "steps back to back, each image read back while the next step renders",
                "latency_ms_per_step": e2e_latency},
        "roofline": {"kernel": {"vertex": "k_cull_groups + k_cull + k_stamp + k_vertex",
                                "stage1": "k_stage1" if algo.get("boxes") else "k_s1cull + k_s1raster"}.get(
                                    rk, f"k_{rk}"), "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": algo[rk], "kernel_ms": t_k,
                     "traffic": read_traffic(rk, wl["name"])},
        # clear, the two frame-cull kernels, the vertex pass (record-culled
        # frames), stage 1 (two kernels when record-culled), stages 2 and 3,
        # the resolve
        "gpu_launches": (7 if algo.get("boxes") else 10) * args.steps,
        "clocks": clk,
    }
    if parity is not None:
        line["parity"] = "bit-exact" if parity_ok else "MISMATCH"
        line["parity_detail"] = parity
    if not args.no_cpu_baseline:
        if oracle_s is not None and len(wl["instances"]) == 1 and oracle_s < 30.0:
            # the parity check's oracle raster of the whole frame is the baseline
            ncores = os.cpu_count() or 1
            line["cpu_baseline"] = {"value": T / oracle_s / 1e9, "unit": "Gtris/s", "cores": ncores, "kind": "port",
                                    "sample": f"oracle raster of the whole frame (all {T:,} triangles), all {ncores} "
                                              f"host threads (OpenMP), {oracle_s:.2f} s"}
        else:
            line["cpu_baseline"] = cpu_baseline(wl)
    if args.sub_results and world == 1 and wl["name"] == DEFAULT_WORKLOAD:
        # the same mesh seen whole from outside: its geometry must be read
        orbit = sub_workload(wl, "planet_orbit_400m_1080p")
        subs = [sub_plain(args, orbit, ctx, handles, True)]
        ctx.close()
        del wl, handles, orbit
        torch.cuda.empty_cache()
        subs += other_sub_results(args)
        line["sub_results"] = subs
        return line
    ctx.close()
    return line


DEFAULT_WORKLOAD = "planet_400m_1080p"
# the other benchmark configurations, timed after the default one when
# --sub-results is on (the default), each against the reference arm's own
SUB_WORKLOADS = ("planet_orbit_400m_1080p", "heightfield_1m_1080p", "instanced_3000x1m_1080p", "batched_64v_60m")


def sub_workload(wl, name):
    """A planet workload on the already built mesh with another camera."""
    import scenes

    out = dict(wl)
    out["name"] = name
    if "orbit" in name:
        out["view"], out["proj"] = scenes.planet_orbit_camera(wl["W"], wl["H"])
        out["desc"] = wl["desc"].replace("camera 0.035 radii above the surface",
                                         "seen whole from 2.6 radii (about half of the triangles face the camera, "
                                         "all of them in the frustum)")
    return out


def other_sub_results(args):
    import torch

    import pycurast as pc

    subs = []
    for name in SUB_WORKLOADS[1:]:
        wl = build_workload(name)
        if wl.get("batched"):
            subs.append(sub_batched(args, wl))
        else:
            ctx = pc.Context()
            handles = [ctx.mesh_from_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
                       if wl["device"] else ctx.mesh_from_host(p, i, c) for (p, i, c) in wl["meshes"]]
            # the 3e9-triangle instanced frame's oracle takes tens of seconds:
            # its parity is checked by the tests at the same size
            subs.append(sub_plain(args, wl, ctx, handles, len(wl["instances"]) == 1))
            ctx.close()
        del wl
        torch.cuda.empty_cache()
    return subs


def sub_plain(args, wl, ctx, handles, with_parity):
    """A compact record of the plain frame of `wl` (meshes resident in HBM,
    `handles` on `ctx`): device-timed steps, the per-stage split, the
    dominant kernel's roofline and the parity of the last frame."""
    import torch

    import pycurast as pc

    T, V, Tu = scene_counts(wl)
    W, H = wl["W"], wl["H"]
    inst = pc.make_instances([(handles[m], w) for m, w in wl["instances"]])
    cam = pc.make_camera(wl["view"], wl["proj"], W, H)
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    flush = None
    if 12 * Tu + 12 * V + 12 * W * H < 2 * L2_BYTES:
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_SYNC, stream=sh)
    for _ in range(max(args.warmup - 1, 0)):
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=0, stream=sh)
    ctx.sync()
    _, fstats = ctx.stats()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        if flush is not None:
            flush.fill_(k)
        evs[k][0].record(stream)
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=0, stream=sh)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    ms_steps = [a.elapsed_time(b) for a, b in evs]
    ms = float(np.mean(ms_steps))
    ctx.drain_stage_times()
    for k in range(args.steps):
        if flush is not None:
            flush.fill_(k)
        ctx.render(inst, cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_TIMING, stream=sh)
    torch.cuda.synchronize()
    ctx.sync()
    stage_ms, nframes = ctx.drain_stage_times()
    stage_ms = {k: v / max(nframes, 1) for k, v in stage_ms.items()}
    peak, peak_kind = load_peaks()
    algo, tri_drawn, v_eval = plain_algorithmic_bytes(wl, fstats, T)
    dominant = max(("vertex", "stage1", "stage2", "stage3", "resolve", "clear"), key=lambda x: stage_ms[x])
    rk = "stage1" if dominant not in algo else dominant
    achieved = algo[rk] / (stage_ms[rk] * 1e-3) / 1e9
    frame_bytes = 12 * T + 12 * V + 28 * W * H
    rec = {"workload": wl["name"], "desc": wl["desc"], "metric": "Gtris/s", "value": T / (ms * 1e-3) / 1e9,
           "unit": "Gtris/s", "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
           "step_ms": step_spread(ms_steps), "triangles": T, "width": W, "height": H,
           "l2": "flushed between steps" if flush is not None else "inputs larger than L2",
           "stage_ms": stage_ms, "dominant_stage": dominant,
           "cull": {"work_items": int(fstats.work_items), "work_items_drawn": int(fstats.work_items_drawn),
                    "vertex_chunks": int(fstats.vertex_chunks),
                    "vertex_chunks_evaluated": int(fstats.vertex_chunks_evaluated),
                    "vertex_slices_evaluated": int(getattr(fstats, "vertex_slices_evaluated", 0)),
                    "stage1_survivors": int(fstats.stage1_survivors), "nontrivial": int(fstats.nontrivial),
                    "huge_tiles": int(fstats.huge_tiles)},
           "roofline": {"kernel": {"vertex": "k_cull_groups + k_cull + k_stamp + k_vertex",
                                   "stage1": "k_stage1" if algo.get("boxes") else "k_s1cull + k_s1raster"}.get(
                                       rk, f"k_{rk}"),
                        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_kind": peak_kind, "algorithmic_bytes": algo[rk], "kernel_ms": stage_ms[rk],
                        "traffic": read_traffic(rk, wl["name"])},
           "frame_roofline": {"bytes": frame_bytes, "achieved_gbs": frame_bytes / (ms * 1e-3) / 1e9,
                              "frac": frame_bytes / (ms * 1e-3) / 1e9 / peak,
                              "note": "reference formula 12T+12V+28P"}}
    if with_parity and not args.no_parity:
        par, _, ok = frame_parity(wl, ctx, inst, vis, rgba)
        rec["parity"] = "bit-exact" if ok else "MISMATCH"
        rec["parity_detail"] = par
    elif not args.no_parity:
        rec["parity"] = ("not checked in this run (the CPU oracle takes tens of seconds on this frame); "
                         "tests/test_bench_sizes_gpu.py checks the same frame bit for bit")
    return rec


def sub_batched(args, wl):
    """A compact record of the batched frame (autotuned plan replayed as a
    CUDA graph) beside the plain per-view loop at identical outputs."""
    import torch

    import pycurast as pc
    import scenes

    cams = wl["cams"]
    nv = len(cams)
    ctx = pc.Context()
    p, i, c = wl["meshes"][0]
    h = ctx.mesh_from_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
    inst = pc.make_instances([(h, scenes.identity())])
    ccams = [pc.make_camera(*cam) for cam in cams]
    vis = [torch.empty(W * H, dtype=torch.int64, device="cuda") for _, _, W, H in cams]
    rgba = [torch.empty(W * H, dtype=torch.int32, device="cuda") for _, _, W, H in cams]
    views = [(ccams[k], vis[k].data_ptr(), rgba[k].data_ptr(), 0) for k in range(nv)]
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    ctx.autotune_batch(inst, views)
    plan = pc.BatchPlan(ctx, inst, views)
    for _ in range(args.warmup):
        plan.launch(sh)
    plan.wait()

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            evs[k][0].record(stream)
            fn()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    steps = max(3, min(args.steps, 10))
    ms_steps = timed(lambda: plan.launch(sh), steps)
    plan.wait()
    batched = [v.cpu().numpy() for v in vis]

    def plain():
        for j in range(nv):
            ctx.render(inst, ccams[j], vis[j].data_ptr(), rgba[j].data_ptr(), 0, pc.CR_DISPLAY_VERTEX_COLORS, 0, sh)

    for j in range(nv):  # synchronous frames first: they size the context's queues for every view
        ctx.render(inst, ccams[j], vis[j].data_ptr(), rgba[j].data_ptr(), flags=pc.CR_RENDER_SYNC, stream=sh)
    plain_steps = timed(plain, max(3, min(args.steps, 5)))
    ctx.sync()
    same = all(np.array_equal(a, v.cpu().numpy()) for a, v in zip(batched, vis))
    plan.close()
    ctx.close()
    ms, plain_ms = float(np.mean(ms_steps)), float(np.mean(plain_steps))
    return {"workload": wl["name"], "desc": wl["desc"], "metric": "views/s", "value": nv / (ms * 1e-3),
            "unit": "views/s", "ms_per_step": ms, "steps": steps, "step_ms": step_spread(ms_steps),
            "plain_loop": {"ms_per_step": plain_ms, "views_per_s": nv / (plain_ms * 1e-3)},
            "speedup_vs_plain_loop": plain_ms / ms,
            "parity": "bit-exact vs the plain loop" if same else "MISMATCH vs the plain loop"}


POST_METRIC = "Mpx/s (EDL + SSAO + 2x supersampled display resolve of a 3840x2160 colorbuffer, per pass)"


def post_colorbuffer_oracle(wl):
    """The workload's colorbuffer from the CPU oracle (host uint64 array)."""
    import oracle_lib as ol

    p, i, c = host_mesh(wl["meshes"][0])
    fr = ol.Frame([(p, i, c, wl["instances"][0][1])], wl["view"])
    fb, _ = ol.raster(fr, wl["W"], wl["H"], wl["proj"][5], nthreads=os.cpu_count() or 1)
    cb, _ = ol.resolve(fr, wl["view"], wl["proj"], wl["W"], wl["H"], fb, nthreads=os.cpu_count() or 1)
    return cb


def post_bytes(wl):
    """Algorithmic bytes of one post pass: occlusion reads the colorbuffer
    (8 B) and writes the 4-byte occlusion per source pixel, the blur reads
    that and writes the 4-byte shade, the display resolve reads the
    colorbuffer and the shade of every source pixel and writes one RGBA8 per
    output pixel (neighbour reads hit in cache)."""
    P = wl["W"] * wl["H"]
    return 12 * P + 8 * P + 12 * P + 4 * wl["outW"] * wl["outH"]


def run_post(args, rank, world, local, wl):
    """One step = one cr_postprocess pass (EDL + SSAO + display resolve) on a
    colorbuffer resident in HBM; the pass's working set (66 MB colorbuffer,
    33 MB occlusion, 33 MB shade) exceeds L2."""
    import torch

    import pycurast as pc

    W, H, oW, oH = wl["W"], wl["H"], wl["outW"], wl["outH"]
    ctx = pc.Context(device=local)
    h = ctx.mesh_from_host(*wl["meshes"][0])
    cam = pc.make_camera(wl["view"], wl["proj"], W, H)
    vis = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    cb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    ctx.render([(h, wl["instances"][0][1])], cam, vis.data_ptr(), rgba.data_ptr(), cb.data_ptr(),
               flags=pc.CR_RENDER_SYNC)
    out = torch.empty(oW * oH, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    # the reference's own build computes the pass with --use_fast_math: the
    # headline runs the library's matching mode, the IEEE pass is timed beside it
    flags = pc.CR_POST_EDL | pc.CR_POST_SSAO | pc.CR_POST_FAST_MATH

    def post(d_cb, fl=flags):
        ctx.postprocess(d_cb, W, H, wl["proj"], out.data_ptr(), fl, mode=pc.CR_POST_DISPLAY, window_width=oW,
                        out_size=(oW, oH), stream=sh)

    for _ in range(args.warmup):
        post(cb.data_ptr())
        post(cb.data_ptr(), flags & ~pc.CR_POST_FAST_MATH)
    torch.cuda.synchronize()
    ieee_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        ieee_evs[k][0].record(stream)
        post(cb.data_ptr(), flags & ~pc.CR_POST_FAST_MATH)
        ieee_evs[k][1].record(stream)
    torch.cuda.synchronize()
    ieee_ms = max_over_ranks(float(np.mean([a.elapsed_time(b) for a, b in ieee_evs])), world)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        evs[k][0].record(stream)
        post(cb.data_ptr())
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop() if clocks else None
    post_steps = [a.elapsed_time(b) for a, b in evs]
    ms = max_over_ranks(float(np.mean(post_steps)), world)

    # end to end: the colorbuffer from pinned host memory, the image back
    host_cb = torch.empty(W * H, dtype=torch.int64, pin_memory=True)
    host_cb.copy_(cb)
    host_out = torch.empty(oW * oH, dtype=torch.int32, pin_memory=True)
    cb2 = torch.empty_like(cb)
    e2e_ms = []
    for k in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cb2.copy_(host_cb, non_blocking=True)
        post(cb2.data_ptr())
        host_out.copy_(out, non_blocking=True)
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e = max_over_ranks(float(np.mean(e2e_ms)), world)
    if rank != 0:
        ctx.close()
        return None
    peak, peak_kind = load_peaks()
    algo = post_bytes(wl)
    achieved = algo / (ms * 1e-3) / 1e9
    line = {
        "metric": POST_METRIC,
        "value": world * W * H / (ms * 1e-3) / 1e6,
        "unit": "Mpx/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "width": W, "height": H, "out_width": oW,
                   "out_height": oH, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (132 MB working set per pass)", "step_ms": step_spread(post_steps),
                   "math": "CR_POST_FAST_MATH (the reference build's --use_fast_math approximations)",
                   "ieee_ms_per_step": ieee_ms},
        "e2e": {"value": world * W * H / (e2e * 1e-3) / 1e6, "unit": "Mpx/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": 8 * W * H, "d2h_bytes_per_step": 4 * oW * oH},
        "roofline": {"kernel": "k_ssao_occlusion + k_ssao_blur + k_post_resolve (one pass)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "algorithmic_bytes": algo, "kernel_ms": ms, "traffic": None,
                     "note": "the occlusion taps (32 scattered depth reads per pixel) bound the pass by L1-to-L2 requests, not HBM"},
        "gpu_launches": 3 * args.steps,
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        import oracle_lib as ol

        hcb = host_cb.numpy().view(np.uint64)
        ncores = os.cpu_count() or 1
        t0 = time.perf_counter()
        ol.post(hcb, W, H, wl["proj"], 1, 1, mode=1, window_width=oW, out_size=(oW, oH), nthreads=ncores)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": W * H / dt / 1e6, "unit": "Mpx/s", "cores": ncores, "kind": "port",
                                "sample": f"the oracle's post pass over the whole colorbuffer, all {ncores} host "
                                          f"threads (OpenMP), {dt:.2f} s"}
    ctx.close()
    return line


def glb_writer_module():
    """The binary glTF writer the glb tests build their files with."""
    tests = os.path.join(ROOT, "tests")
    if tests not in sys.path:
        sys.path.insert(0, tests)
    import glb_writer

    return glb_writer


def glb_file(wl):
    glb_writer = glb_writer_module()
    import scenes

    pos, idx, col = scenes.heightfield()
    rgba = col.view(np.uint8).reshape(-1, 4)
    prim = dict(positions=pos, indices=idx, index_type="u32", colors=rgba, color_format="vec4u8")
    n = wl["primitives"]
    nodes = [dict(mesh=k, matrix=scenes.translate_scale(1.1 * (k % 8), 0.0, 0.6 * (k // 8))) for k in range(n)]
    return glb_writer.build_glb([[prim] for _ in range(n)], nodes), idx.shape[0] * n


def h2d_peak_gbs():
    """Pinned host -> device copy rate of this box (1 GiB), the bound of any
    ingest that ends on the device."""
    import torch

    src = torch.empty(1 << 30, dtype=torch.uint8, pin_memory=True)
    dst = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(3):
        dst.copy_(src, non_blocking=True)
    b.record()
    b.synchronize()
    return 3 * (1 << 30) / (a.elapsed_time(b) * 1e-3) / 1e9


GLB_METRIC = "Mtris/s (binary glTF in host memory -> resident meshes + instance list)"


def run_glb(args, rank, world, local, wl):
    """One step = cr_glb_open of the file's bytes, cr_glb_create_meshes (host
    copies uploaded) and cr_glb_instances, ended by a device synchronize.  A
    host-driven path: timed by the host clock with the device synchronized on
    both sides."""
    import torch

    import pycurast as pc

    data, T = glb_file(wl)
    ctx = pc.Context(device=local)

    def step():
        with pc.Glb(data=data) as g:
            handles = g.create_meshes(ctx)
            g.instances(handles)
        torch.cuda.synchronize()
        return handles

    for _ in range(args.warmup):
        for hm in step():
            ctx.mesh_destroy(hm)
    barrier(world)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        hs = step()
        times.append(time.perf_counter() - t0)
        for hm in hs:
            ctx.mesh_destroy(hm)
    barrier(world)
    ms = max_over_ranks(float(np.mean(times)) * 1e3, world)
    # three more steps, each split into its phases (host clock, device
    # synchronized); the median of each phase
    split = []
    for _ in range(3):
        t0 = time.perf_counter()
        g = pc.Glb(data=data)
        t1 = time.perf_counter()
        hs = g.create_meshes(ctx)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        g.instances(hs)
        g.close()
        t3 = time.perf_counter()
        for hm in hs:
            ctx.mesh_destroy(hm)
        split.append(((t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3))
    med = np.median(np.array(split), axis=0)
    phases = {"open": float(med[0]), "create_meshes": float(med[1]), "instances_close": float(med[2])}
    if rank != 0:
        ctx.close()
        return None
    peak = h2d_peak_gbs()
    achieved = len(data) / (ms * 1e-3) / 1e9
    value = world * T / (ms * 1e-3) / 1e6
    line = {
        "metric": GLB_METRIC,
        "value": value,
        "unit": "Mtris/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "triangles": T, "file_bytes": len(data),
                   "parallelism": f"replicas x{world}", "l2": "not applicable (host path; file > L2)",
                   "phases_ms": phases, "step_ms": step_spread([t * 1e3 for t in times])},
        "e2e": {"value": value, "unit": "Mtris/s", "ms_per_step": ms, "h2d_bytes_per_step": len(data),
                "d2h_bytes_per_step": 0},
        "roofline": {"kernel": "host parse + upload (cr_glb_open, cr_glb_create_meshes)", "bound": "pcie",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": "measured here: pinned host-to-device copy of 1 GiB",
                     "algorithmic_bytes": len(data), "kernel_ms": ms, "traffic": None},
        "gpu_launches": None,
        "note": "the step is host code plus one upload and one mesh-preparation pass per primitive",
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = glb_oracle_baseline(wl)
    ctx.close()
    return line


def glb_oracle_baseline(wl):
    """The oracle's restatement of the reference loader (Python, one thread)
    on one primitive of the same form."""
    glb_writer = glb_writer_module()
    import scenes

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import glb_oracle

    pos, idx, col = scenes.heightfield()
    prim = dict(positions=pos, indices=idx, index_type="u32", colors=col.view(np.uint8).reshape(-1, 4),
                color_format="vec4u8")
    sample = glb_writer.build_glb([[prim]], [dict(mesh=0, matrix=scenes.identity())])
    t0 = time.perf_counter()
    glb_oracle.load(sample)
    dt = time.perf_counter() - t0
    return {"value": idx.shape[0] / dt / 1e6, "unit": "Mtris/s", "cores": 1, "kind": "port",
            "sample": f"the oracle's loader restatement on a one-primitive file of the same form "
                      f"({idx.shape[0]:,} triangles), one thread, {dt:.2f} s"}


def run_batched(args, rank, world, local, wl):
    """One step = one batched frame of all views (the autotuned plan replayed
    as a CUDA graph: table upload, clear, vertex pass, stages 1-3, resolve).
    The same views rendered one cr_render at a time are timed beside it."""
    import torch

    import pycurast as pc

    T, V, Tu = scene_counts(wl)
    cams = wl["cams"]
    nv = len(cams)
    P = sum(W * H for _, _, W, H in cams)
    ctx = pc.Context(device=local)
    p, i, c = wl["meshes"][0]
    h = ctx.mesh_from_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
    inst = pc.make_instances([(h, scenes_identity())])
    ccams = [pc.make_camera(*cam) for cam in cams]
    vis = [torch.empty(W * H, dtype=torch.int64, device="cuda") for _, _, W, H in cams]
    rgba = [torch.empty(W * H, dtype=torch.int32, device="cuda") for _, _, W, H in cams]
    host_rgba = [torch.empty(W * H, dtype=torch.int32, pin_memory=True) for _, _, W, H in cams]
    views = [(ccams[k], vis[k].data_ptr(), rgba[k].data_ptr(), 0) for k in range(nv)]
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    # autotune this scene class, then capture the frame as a graph
    t0 = time.perf_counter()
    tuning = ctx.autotune_batch(inst, views)
    tune_s = time.perf_counter() - t0
    plan = pc.BatchPlan(ctx, inst, views)
    for _ in range(args.warmup):
        plan.launch(sh)
    fstats = plan.wait()

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            evs[k][0].record(stream)
            fn(k)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    # ---- device-timed region (visbuffers + images are ~2 GB: inputs and
    # outputs far larger than L2) ------------------------------------------
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ms_steps = timed(lambda k: plan.launch(sh), args.steps)
    barrier(world)
    clk = clocks.stop() if clocks else None
    plan.wait()
    ms = max_over_ranks(float(np.mean(ms_steps)), world)

    # per-stage device times of the batched frame (eager, same shapes)
    ctx.drain_stage_times()
    for _ in range(3):
        ctx.render_batch(inst, views, pc.CR_DISPLAY_VERTEX_COLORS, pc.CR_RENDER_TIMING, sh)
    stage_ms, nfr = ctx.drain_stage_times()
    stage_ms = {k: v / max(nfr, 1) for k, v in stage_ms.items()}

    # ---- the plain per-view loop on the same GPU ---------------------------
    def plain(k, flags=0):
        for j in range(nv):
            ctx.render(inst, ccams[j], vis[j].data_ptr(), rgba[j].data_ptr(), 0, pc.CR_DISPLAY_VERTEX_COLORS,
                       flags, sh)

    plain(0, pc.CR_RENDER_SYNC)
    plain_steps = max(3, min(args.steps, 5))
    plain_ms = max_over_ranks(float(np.mean(timed(plain, plain_steps))), world)

    # ---- end to end: cameras in (graph's table upload), 64 RGBA8 images out
    barrier(world)
    torch.cuda.synchronize()

    def e2e_step(k):
        plan.launch(sh)
        for j in range(nv):
            host_rgba[j].copy_(rgba[j], non_blocking=True)

    e2e_ms = timed(e2e_step, max(3, min(args.steps, 5)))
    plan.wait()
    e2e = max_over_ranks(float(np.mean(e2e_ms)), world)
    plan.close()
    if rank != 0:
        ctx.close()
        return None
    peak, peak_kind = load_peaks()
    # algorithmic bytes: vertex pass 12 B position read + 48 B record write per
    # vertex; stage 1 12 B index tile per triangle + each 48 B record once;
    # whole frame 12T + 12V (geometry once for all views) + 28 B per pixel of
    # every view (visbuffer clear and write-back, resolve read + RGBA8 write)
    algo = {"vertex": 60 * V, "stage1": 12 * T + 48 * V}
    dominant = max(("vertex", "stage1", "stage2", "stage3", "resolve", "clear"), key=lambda s: stage_ms[s])
    rk = "stage1" if dominant not in algo else dominant
    t_k = stage_ms[rk]
    achieved = algo[rk] / (t_k * 1e-3) / 1e9
    frame_bytes = 12 * T + 12 * V + 28 * P
    line = {
        "metric": "views/s (batched frame of 64 views of uneven resolution, one CUDA-graph launch per step)",
        "value": world * nv / (ms * 1e-3),
        "unit": "views/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "triangles": T, "vertices": V, "views": nv,
                   "pixels": P, "parallelism": f"replicas x{world}",
                   "l2": "per-step visbuffers and images ({:.1f} GB) exceed L2".format(28 * P / 1e9),
                   "stage_ms": stage_ms, "dominant_stage": dominant, "step_ms": step_spread(ms_steps),
                   "nontrivial": int(fstats.nontrivial), "huge_tiles": int(fstats.huge_tiles),
                   "plain_loop": {"ms_per_step": plain_ms, "views_per_s": world * nv / (plain_ms * 1e-3),
                                  "note": f"{nv} cr_render calls per step, same GPU, same outputs"},
                   "speedup_vs_plain_loop": plain_ms / ms,
                   "tuning": {"seconds": tune_s, "candidates": int(tuning.candidates),
                              "ms_default_shapes": float(tuning.ms_before), "ms_tuned": float(tuning.ms_after),
                              "vertex_blocks": int(tuning.vertex_blocks), "stage1": [int(tuning.stage1_blocks),
                                                                                    int(tuning.stage1_warps)],
                              "stage2": [int(tuning.stage2_blocks), int(tuning.stage2_warps)],
                              "stage3_blocks": int(tuning.stage3_blocks)},
                   "frame_roofline": {"bytes": frame_bytes, "achieved_gbs": frame_bytes / (ms * 1e-3) / 1e9,
                                      "frac": frame_bytes / (ms * 1e-3) / 1e9 / peak}},
        "e2e": {"value": world * nv / (e2e * 1e-3), "unit": "views/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 4 * P},
        "roofline": {"kernel": f"k_{rk}_views", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "algorithmic_bytes": algo[rk],
                     "kernel_ms": t_k, "traffic": read_traffic(rk + "_views", wl["name"])},
        "gpu_launches": 6 * args.steps,
        "clocks": clk,
    }
    ctx.close()
    return line


def served_requests(n, rate, seed=53):
    """Seeded request stream: arrival times (Poisson), scene 0-2, camera."""
    import math

    import scenes

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    tcams = scenes.batch_cameras(256, seed=seed + 1)
    for k in range(n):
        W, H = scenes.BATCH_RESOLUTIONS[int(rng.integers(4))]
        proj = scenes.perspective(60.0, W / H, 0.001, 10.0)
        s = int(rng.integers(3))
        if s == 0:  # heightfield: around the benchmark camera
            eye = np.array([0.5, 0.6, 0.45]) + rng.uniform(-0.15, 0.15, 3)
            view = scenes.look_at(eye, (0.5 + rng.uniform(-0.1, 0.1), 0.0, 0.24))
        elif s == 1:  # terrain: the batched-views camera set
            view = tcams[int(rng.integers(len(tcams)))][0]
        else:  # planet: the benchmark camera turned by a few degrees
            v0, _ = scenes.planet_camera(W, H)
            a, b = rng.uniform(-0.05, 0.05, 2)
            R = np.eye(4)
            R[:3, :3] = (np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]]) @
                         np.array([[1, 0, 0], [0, math.cos(b), -math.sin(b)], [0, math.sin(b), math.cos(b)]]))
            view = (R.T @ np.asarray(v0, np.float64).reshape(4, 4).T).T.reshape(16).astype(np.float32)
        out.append((float(t[k]), s, view, proj, W, H))
    return out


def run_served(args, rank, world, local, wl):
    """Continuous batching at the configured Poisson rate (latency), then the
    same kind of requests submitted at once (capacity), then the plain loop:
    one cr_render per request.  Beside them, frames of the out-of-core scene
    run on the server's out-of-core lane."""
    import torch

    import pycurast as pc
    import scenes

    rate = wl["rate"]
    ctx = pc.Context(device=local)
    t0 = time.perf_counter()
    hf = scenes.heightfield()
    tp, ti, tc = scenes.terrain(n=5477, device="cuda")
    pp, pi, pcol = scenes.planet(400_000_000, device="cuda")
    h_hf = ctx.mesh_from_host(*hf)
    h_tr = ctx.mesh_from_device(tp.data_ptr(), tp.shape[0], ti.data_ptr(), ti.shape[0], tc.data_ptr())
    h_pl = ctx.mesh_from_device(pp.data_ptr(), pp.shape[0], pi.data_ptr(), pi.shape[0], pcol.data_ptr())
    insts = [[(h_hf, scenes.identity())], [(h_tr, scenes.identity())], [(h_pl, scenes.identity())]]
    tris = [hf[1].shape[0], ti.shape[0], pi.shape[0]]
    nodes, okeep = scenes.ooc_terrain(nodes_x=args.ooc_nodes, nodes_z=args.ooc_nodes)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    ooc = pc.OocScene(ctx, nodes, geometry_budget=32 << 30)
    ocams = [pc.make_camera(*c) for c in scenes.ooc_cameras(64)]
    ooc_tris = sum(n[4] for n in nodes)

    def serve(srv, ids, oid, reqs, paced, with_ooc):
        srv.reset_stats()
        start = time.perf_counter()
        pending = set()
        k = 0
        ook = 0
        last_ooc = 0.0
        while k < len(reqs) or pending:
            now = time.perf_counter() - start
            while k < len(reqs) and (not paced or reqs[k][0] <= now):
                _, s, view, proj, W, H = reqs[k]
                pending.add(srv.submit(ids[s], pc.make_camera(view, proj, W, H)))
                k += 1
            if with_ooc and k < len(reqs) and now - last_ooc > 0.25:  # out-of-core frames beside them
                pending.add(srv.submit(oid, ocams[ook % len(ocams)]))
                ook += 1
                last_ooc = now
            for r in srv.poll():
                if r.status != pc.CR_OK:
                    raise RuntimeError(f"request {r.ticket} failed: {r.status}")
                srv.release(r.ticket)
                pending.discard(r.ticket)
            if paced and k < len(reqs):
                time.sleep(max(0.0, min(0.0005, reqs[k][0] - (time.perf_counter() - start))))
            else:
                time.sleep(0.0002)
        return srv.stats(), time.perf_counter() - start, ook

    n_req = max(200, int(rate * args.serve_seconds))
    reqs = served_requests(n_req, rate)
    cap_reqs = served_requests(args.capacity_requests, rate, seed=61)
    # one long-lived server: a warm-up burst (its slots' scratch and each
    # scene's queue demand reach steady state), then the capacity burst, then
    # the paced run with out-of-core frames beside it
    with pc.Server(ctx, memory_budget=64 << 30, slots=3) as srv:
        ids = [srv.add_scene(s) for s in insts]
        oid = srv.add_ooc_scene(ooc)
        serve(srv, ids, oid, served_requests(args.capacity_requests, rate, seed=59), False, False)
        st_cap, wall_cap, _ = serve(srv, ids, oid, cap_reqs, False, False)
        st_paced, wall_paced, n_ooc = serve(srv, ids, oid, reqs, True, True)

    # the plain loop: the capacity requests one cr_render at a time
    vis = torch.empty(3840 * 2160, dtype=torch.int64, device="cuda")
    rgba = torch.empty(3840 * 2160, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    for _, s, view, proj, W, H in cap_reqs[:8]:
        ctx.render(insts[s], pc.make_camera(view, proj, W, H), vis.data_ptr(), rgba.data_ptr(), flags=0,
                   stream=stream.cuda_stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _, s, view, proj, W, H in cap_reqs:
        ctx.render(insts[s], pc.make_camera(view, proj, W, H), vis.data_ptr(), rgba.data_ptr(), flags=0,
                   stream=stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    plain_s = a.elapsed_time(b) * 1e-3
    plain_vps = len(cap_reqs) / plain_s
    # one out-of-core frame alone, cold and warm cache
    ooc_stats = []
    for cam in ocams[:2] + ocams[:1]:
        c0 = time.perf_counter()
        st = ooc.render(cam, vis.data_ptr(), rgba.data_ptr(), flags=pc.CR_RENDER_SYNC) if cam.width * cam.height <= 3840 * 2160 else None
        ooc_stats.append({"ms": (time.perf_counter() - c0) * 1e3, "visible_nodes": st.visible_nodes,
                          "visible_triangles": st.visible_triangles, "uploaded_nodes": st.uploaded_nodes,
                          "uploaded_GB": st.uploaded_bytes / 1e9, "resident_hits": st.resident_hits,
                          "passes": st.passes})
    ooc.close()
    ctx.close()
    if rank != 0:
        return None
    return {
        "metric": "views/s served (continuous batching, mixed scenes and resolutions), p50/p99 latency vs plain loop",
        "value": world * st_cap.views_per_s,
        "unit": "views/s",
        "n_gpus": world,
        "steps": len(cap_reqs),
        "warmup": 64,
        "ms_per_step": 1e3 / st_cap.views_per_s,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "scene_triangles": tris,
                   "ooc": {"nodes": len(nodes), "triangles": ooc_tris, "host_bytes": int(okeep[0].numel() * 4 +
                                                                                     okeep[1].numel() * 4),
                           "geometry_budget": 32 << 30, "frames_beside_paced_run": n_ooc, "alone": ooc_stats},
                   "paced": {"rate_per_s": rate, "requests": len(reqs), "wall_s": wall_paced,
                             "views_per_s": st_paced.views_per_s, "p50_ms": st_paced.p50_ms,
                             "p99_ms": st_paced.p99_ms, "mean_ms": st_paced.mean_ms,
                             "batches": int(st_paced.batches), "peak_GB": st_paced.peak_bytes / 1e9},
                   "capacity": {"requests": len(cap_reqs), "views_per_s": st_cap.views_per_s,
                                "p50_ms": st_cap.p50_ms, "p99_ms": st_cap.p99_ms, "batches": int(st_cap.batches),
                                "mean_batch": st_cap.batched_views / max(1, st_cap.batches)},
                   "plain_loop": {"views_per_s": plain_vps, "seconds": plain_s,
                                  "note": "the capacity requests, one cr_render each, same GPU"},
                   "speedup_vs_plain_loop": st_cap.views_per_s / plain_vps,
                   "setup_s": setup_s, "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * st_cap.views_per_s, "unit": "views/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0, "note": "host submit to device completion, results left on the device"},
        "gpu_launches": None,
        "clocks": None,
    }


def scenes_identity():
    import scenes

    return scenes.identity()


# ---------------------------------------------------------------------------
# the reference's own kernels
# ---------------------------------------------------------------------------
def run_reference(args, rank, world, local):
    if rank != 0:
        return None
    import oracle_lib as ol

    wl = build_workload(args.workload)
    if wl.get("batched"):
        return run_reference_batched(args, wl, local)
    if wl.get("post"):
        return run_reference_post(args, wl, local)
    if wl.get("glb"):
        # the reference loader does not build here (C++23 <print>/<stacktrace>,
        # its mapped-file layer, scene graph and CUDA driver): its restatement
        # is the reference arm
        base = glb_oracle_baseline(wl)
        return {"impl": "reference", "metric": GLB_METRIC, "value": base["value"], "unit": "Mtris/s", "n_gpus": 1,
                "steps": 1, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
                "config": {"workload": wl["name"], "desc": wl["desc"], "parallelism": "single host thread"},
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "Mtris/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        ref = ol.Reference("native", device=local)
    except Exception as e:  # noqa: BLE001
        return {"impl": "reference", "unavailable": f"reference kernels not loadable: {e}"}
    r = ref_plain(args, wl, ref)
    line = {
        "impl": "reference",
        "metric": "Gtris/s @1080p (plain 3-stage visbuffer + resolve, one frame per step)",
        "value": r["value"],
        "unit": "Gtris/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "triangles": r["triangles"], "vertices": r["vertices"],
                   "width": wl["W"], "height": wl["H"], "parallelism": "single GPU", "stage_ms": r["stage_ms"],
                   "nontrivial": r["nontrivial"], "huge_tiles": r["huge_tiles"],
                   "build": "CuRast NVRTC recipe (--use_fast_math, LTO) for sm_100a"},
        "cpu_baseline": {"kind": "reference", "value": r["value"], "unit": "Gtris/s", "cores": 0,
                         "sample": "not a CPU run: the reference has no CPU rasterizer, so its own CUDA kernels "
                                   "are timed on this B200 (whole frame)"},
        "e2e": {"value": r["value"], "unit": "Gtris/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.sub_results and wl["name"] == DEFAULT_WORKLOAD:
        import torch

        subs = [ref_plain(args, sub_workload(wl, "planet_orbit_400m_1080p"), ref, ids=r["ids"])]
        ref.reset()
        del wl
        torch.cuda.empty_cache()
        for name in SUB_WORKLOADS[1:]:
            sw = build_workload(name)
            if sw.get("batched"):
                b = run_reference_batched(args, sw, local, ref=ref)
                subs.append({"workload": name, "desc": sw["desc"], "metric": "views/s", "value": b["value"],
                             "unit": "views/s", "ms_per_step": b["ms_per_step"], "steps": b["steps"]})
            else:
                subs.append(ref_plain(args, sw, ref))
            ref.reset()
            del sw
            torch.cuda.empty_cache()
        for x in subs:
            x.pop("ids", None)
        line["sub_results"] = subs
    return line


def ref_plain(args, wl, ref, ids=None):
    """The reference's own kernels (native build) on the plain frame of `wl`:
    the mean device time of args.steps frames (clear + stages 1-3, then the
    resolve), queues sized from the CPU oracle's exact counts with a margin
    (the reference never checks its capacities)."""
    import oracle_lib as ol

    T, V, Tu = scene_counts(wl)
    W, H = wl["W"], wl["H"]
    if ids is None:
        if wl.get("compressed"):  # the reference's *_compressed kernels
            ids = [ref.mesh_compressed_host(cp.packed, cp.positions, cp.num_triangles, dec[2], cp.aabb_min,
                                            cp.aabb_max, cp.index_min, cp.index_max)
                   for cp, dec in zip(wl["compressed"], wl["decoded"])]
        elif wl["device"]:
            ids = [ref.mesh_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
                   for (p, i, c) in wl["meshes"]]
        else:
            ids = [ref.mesh_host(p, i, c) for (p, i, c) in wl["meshes"]]
    mids = [ids[m] for m, _ in wl["instances"]]
    worlds = np.stack([np.asarray(w, np.float32).reshape(16) for _, w in wl["instances"]])
    meshes = wl["decoded"] if wl.get("compressed") else [host_mesh(m) for m in wl["meshes"]]
    items = [(*meshes[m], w) for m, w in wl["instances"]]
    _, ost = ol.raster(ol.Frame(items, wl["view"]), W, H, wl["proj"][5], nthreads=os.cpu_count() or 1)
    del items, meshes
    cap_nt = min(T, 2 * int(ost.nontrivial) + (1 << 20))
    cap_huge = 2 * int(ost.huge_tiles) + (1 << 20)
    ref.frame(mids, worlds, wl["view"], wl["proj"], W, H, instanced=True, cap_nontrivial=cap_nt,
              cap_huge=cap_huge, frames=max(args.warmup, 1), want_color=False)
    _, _, _, ms, counts = ref.frame(mids, worlds, wl["view"], wl["proj"], W, H, instanced=True,
                                    cap_nontrivial=cap_nt, cap_huge=cap_huge, frames=args.steps, want_color=False)
    step_ms = float(ms[0] + ms[1])
    return {"workload": wl["name"], "desc": wl["desc"], "metric": "Gtris/s", "value": T / (step_ms * 1e-3) / 1e9,
            "unit": "Gtris/s", "ms_per_step": step_ms, "steps": args.steps, "triangles": T, "vertices": V,
            "stage_ms": {"clear+raster": float(ms[0]), "resolve": float(ms[1])},
            "nontrivial": int(counts[0]), "huge_tiles": int(counts[1]), "ids": ids}


def run_reference_batched(args, wl, local, ref=None):
    """The reference renders one view per CuRast::draw: its own kernels run
    once per view (same cameras, resolutions and mesh); a step is all views."""
    import oracle_lib as ol

    T, V, Tu = scene_counts(wl)
    cams = wl["cams"]
    if ref is None:
        try:
            ref = ol.Reference("native", device=local)
        except Exception as e:  # noqa: BLE001
            return {"impl": "reference", "unavailable": f"reference kernels not loadable: {e}"}
    p, i, c = wl["meshes"][0]
    mid = ref.mesh_device(p.data_ptr(), p.shape[0], i.data_ptr(), i.shape[0], c.data_ptr())
    hp, hi, hc = host_mesh(wl["meshes"][0])
    world = np.asarray(wl["instances"][0][1], np.float32).reshape(1, 16)
    total_ms = 0.0
    steps = max(1, min(args.steps, 5))
    for view, proj, W, H in cams:
        # the reference never checks its queue capacities: size them from the
        # CPU oracle's exact counts for this view, with a wide margin
        _, ost = ol.raster(ol.Frame([(hp, hi, hc, world[0])], view), W, H, proj[5], nthreads=os.cpu_count() or 1)
        cap_nt = min(T, 2 * int(ost.nontrivial) + (1 << 20))
        cap_huge = 2 * int(ost.huge_tiles) + (1 << 20)
        ref.frame([mid], world, view, proj, W, H, instanced=True, cap_nontrivial=cap_nt, cap_huge=cap_huge,
                  frames=1, want_color=False)
        _, _, _, ms, _ = ref.frame([mid], world, view, proj, W, H, instanced=True, cap_nontrivial=cap_nt,
                                   cap_huge=cap_huge, frames=steps, want_color=False)
        total_ms += float(ms[0] + ms[1])
    v = len(cams) / (total_ms * 1e-3)
    return {
        "impl": "reference",
        "metric": "views/s (batched frame of 64 views of uneven resolution, one CUDA-graph launch per step)",
        "value": v,
        "unit": "views/s",
        "n_gpus": 1,
        "steps": steps,
        "warmup": 1,
        "ms_per_step": total_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "triangles": T, "vertices": V, "views": len(cams),
                   "parallelism": "single GPU",
                   "build": "CuRast NVRTC recipe (--use_fast_math, LTO) for sm_100a; one frame per view"},
        "cpu_baseline": {"kind": "reference", "value": v, "unit": "views/s", "cores": 0,
                         "sample": "not a CPU run: the reference's own CUDA kernels, one frame per view"},
        "e2e": {"value": v, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference_post(args, wl, local):
    """The reference's own post kernels (NVRTC fast-math build) on the same
    colorbuffer, repeated back to back."""
    import oracle_lib as ol

    try:
        ref = ol.Reference("native", device=local)
    except Exception as e:  # noqa: BLE001
        return {"impl": "reference", "unavailable": f"reference kernels not loadable: {e}"}
    W, H, oW, oH = wl["W"], wl["H"], wl["outW"], wl["outH"]
    cb = post_colorbuffer_oracle(wl)
    ref.post_timed(cb, W, H, wl["proj"], 1, 1, max(args.warmup, 1), mode=1, window_width=oW, out_size=(oW, oH))
    ms, _ = ref.post_timed(cb, W, H, wl["proj"], 1, 1, args.steps, mode=1, window_width=oW, out_size=(oW, oH))
    v = W * H / (ms * 1e-3) / 1e6
    return {
        "impl": "reference",
        "metric": POST_METRIC,
        "value": v,
        "unit": "Mpx/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "desc": wl["desc"], "width": W, "height": H, "out_width": oW,
                   "out_height": oH, "parallelism": "single GPU",
                   "build": "CuRast NVRTC recipe (--use_fast_math, LTO) for sm_100a"},
        "cpu_baseline": {"kind": "reference", "value": v, "unit": "Mpx/s", "cores": 0,
                         "sample": "not a CPU run: the reference's own CUDA post kernels on this B200"},
        "e2e": {"value": v, "unit": "Mpx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    help="planet_400m_1080p (the 400M-triangle dense mesh), planet_<N>m_1080p, heightfield_1m_1080p, "
                         "instanced_<K>x<N>m_1080p, batched_<V>v_<N>m (V cameras over an N-million-triangle "
                         "terrain), served_<R>rps, post_2160p_ss2 (EDL + SSAO + supersampled resolve), glb_<N>m "
                         "(binary glTF ingest of N one-million-triangle primitives)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the last frame")
    ap.add_argument("--no-sub-results", dest="sub_results", action="store_false",
                    help="the default workload's line omits the other configurations")
    ap.add_argument("--ooc-nodes", type=int, default=247, help="out-of-core scene: nodes per side (served_*)")
    ap.add_argument("--serve-seconds", type=float, default=4.0, help="paced serving run length (served_*)")
    ap.add_argument("--capacity-requests", type=int, default=512, help="requests of the capacity run (served_*)")
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
