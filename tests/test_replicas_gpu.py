"""Replicas rendering through the library: two processes (gloo process
group, as bench.py's plumbing), each with its own context on the GPU it is
given (with one GPU both share it: the replicas never wait on each other in
a kernel, only at host barriers), each rendering its own view of the same
seeded scene and checking it bit for bit against the CPU oracle; the job's
time is the max over the ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "curast-ooc_b200"), os.path.join(ROOT, "oracle")]
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import bench
    import oracle_lib as ol
    import pycurast as pc
    import scenes

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        device = rank % torch.cuda.device_count()
        torch.cuda.set_device(device)
        W, H = 320, 180
        pos, idx, col = scenes.heightfield(nx=96, nz=48, seed=3 + rank)
        view, proj = scenes.heightfield_camera(W, H)
        with pc.Context(device=device) as ctx:
            h = ctx.mesh_from_host(pos, idx, col)
            vis = torch.empty(W * H, dtype=torch.int64, device=f"cuda:{device}")
            rgba = torch.empty(W * H, dtype=torch.int32, device=f"cuda:{device}")
            cam = pc.make_camera(view, proj, W, H)
            bench.barrier(world)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            ctx.render([(h, scenes.identity())], cam, vis.data_ptr(), rgba.data_ptr())
            b.record()
            torch.cuda.synchronize()
            worst = bench.max_over_ranks(a.elapsed_time(b), world)
            got = vis.cpu().numpy().view(np.uint64)
        want, _ = ol.raster(ol.Frame([(pos, idx, col, scenes.identity())], view), W, H, proj[5])
        bad = int((got != want).sum())
        bench.barrier(world)
        out.put((rank, bad, int((got != pc.CLEAR_PIXEL).sum()), worst))
    finally:
        dist.destroy_process_group()


def test_two_replicas_render_and_match_the_oracle(gpu):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(world))
    worst = {r[3] for r in res}
    assert len(worst) == 1  # every rank reports the same max over ranks
    for rank, bad, covered, _ in res:
        assert bad == 0, f"rank {rank}: {bad} pixels differ from the oracle"
        assert covered > 1000
