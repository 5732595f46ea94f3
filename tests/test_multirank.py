"""The multi-GPU plumbing on CPU: two ranks with the gloo backend (rendezvous on
127.0.0.1).  Replicas render distinct frames of the workload, batches of views
shard without overlap, timings reduce to the max over ranks, and the reference
arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, queue):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "black-hole_b200")]
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        import bench
        from bhrt import lib, ranks, scenes
        cams = [tuple(P.camPos.tolist()) for P in bench.workload(lib.derive, rank)]
        all_times = [None] * world
        dist.all_gather_object(all_times, cams)
        reduced = ranks.max_over_ranks([float(rank), 10.0 - rank, 3.5], world)
        views = scenes.batch_views(lib.derive, 16, 1234)
        mine = ranks.shard_views(list(range(len(views))), rank, world)
        all_shards = [None] * world
        dist.all_gather_object(all_shards, mine)
        if rank == 0:
            queue.put((all_times, reduced, all_shards))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    all_times, reduced, all_shards = queue.get()
    # distinct orbit frames per replica: no camera position rendered by both ranks
    assert len(all_times[0]) == len(all_times[1]) == 30
    assert not set(all_times[0]) & set(all_times[1])
    assert reduced == [1.0, 10.0, 3.5]                               # max over ranks
    assert sorted(all_shards[0] + all_shards[1]) == list(range(16))  # every view once
    assert not set(all_shards[0]) & set(all_shards[1])


def test_shard_views_bounds():
    sys.path.insert(0, os.path.join(ROOT, "black-hole_b200"))
    from bhrt import ranks
    assert ranks.shard_views(list(range(5)), 1, 3) == [1, 4]
    with pytest.raises(ValueError):
        ranks.shard_views([1], 2, 2)
    # orbit frames: 8 ranks of 30 frames out of 300 never share a frame
    seen = [ranks.orbit_frames_for_rank(300, 30, r) for r in range(8)]
    flat = [k for fr in seen for k in fr]
    assert len(flat) == len(set(flat)) == 240 and all(0 <= k < 300 for k in flat)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
