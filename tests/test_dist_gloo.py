"""Host logic of the multi-GPU sweep with world_size-2 gloo ranks on CPU
(the solve routine is a fake: no GPU, no collective on the solve path)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cugmres_b200 import dist as D


def test_shard_systems_is_a_balanced_partition():
    rng = np.random.default_rng(0)
    sizes = list(rng.choice([96, 128, 192, 256, 384, 512], size=257))
    for world in (1, 2, 3, 8):
        parts = [D.shard_systems(sizes, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(int(sizes[i]) ** 2 for i in p) for p in parts]
        assert max(loads) - min(loads) <= 512 ** 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = [dict(g_block=np.zeros((n, n))) for n in (96, 512, 128, 256, 384, 96, 192)]

        def fake_solve(batch):
            return [dict(status=0 if s["g_block"].shape[0] < 400 else 3, iterations=s["g_block"].shape[0],
                         seconds=s["g_block"].shape[0] / 1000.0, rel_residual_true=1e-11) for s in batch]

        recs, stats = D.run_sweep(systems, rank, world, fake_solve, timer=lambda: 1.0 + rank)
        q.put((rank, [r["index"] for r in recs], stats))
    finally:
        dist.destroy_process_group()


def test_sweep_gather_and_max_timing_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, idx, stats in out:
        assert idx == list(range(7))              # every rank sees every record
        assert stats["systems"] == 7
        assert stats["converged"] == 6            # the N = 512 system "failed"
        assert stats["wall_s"] == 2.0             # max over ranks of 1.0 and 2.0
        assert stats["iterations_total"] == 96 + 512 + 128 + 256 + 384 + 96 + 192
