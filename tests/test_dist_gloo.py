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


def _oracle_worker(rank, world, port, q):
    """Each rank solves its share with the CPU oracle's GMRES(m) (a real solve,
    standing in for the GPU bucket call) through the same run_sweep path."""
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import oracle as O
    from oracle import problems as OP
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        O.set_threads(1)
        systems = [OP.helmholtz(n, e, seed=s) for n, e, s in ((16, 2.25, 1), (24, 4.0, 2), (12, 2.0, 3), (20, 3.0, 4),
                                                              (16, 6.0, 5))]

        def oracle_solve(batch):
            out = []
            for s in batch:
                gh = O.spectrum(s["g_block"], OP.embedding(s["N"]))
                o = O.gmres(gh, s["chi"] * s["chi_scale"], s["b"], restart=20, maxiter=200, tol=1e-10)
                out.append(dict(status=o["status"], iterations=o["iterations"], cycles=o["cycles"], seconds=0.0,
                                rel_residual_true=o["true_res"]))
            return out

        recs, stats = D.run_sweep(systems, rank, world, oracle_solve)
        q.put((rank, recs, stats))
    finally:
        dist.destroy_process_group()


def test_sweep_of_real_oracle_solves_over_two_gloo_ranks():
    """Shards of real solves: every record comes back to every rank, equal to
    the same system solved alone, and each system was solved by exactly one rank."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import oracle as O
    from oracle import problems as OP
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [16, 24, 12, 20, 16]
    owners = [D.shard_systems(sizes, r, 2) for r in range(2)]
    assert sorted(owners[0] + owners[1]) == list(range(5)) and owners[0] and owners[1]
    for rank, recs, stats in out:
        assert [r["index"] for r in recs] == list(range(5))
        assert stats["systems"] == 5
        for r, (n, e, s) in zip(recs, ((16, 2.25, 1), (24, 4.0, 2), (12, 2.0, 3), (20, 3.0, 4), (16, 6.0, 5))):
            pr = OP.helmholtz(n, e, seed=s)
            o = O.gmres(O.spectrum(pr["g_block"], OP.embedding(n)), pr["chi"] * pr["chi_scale"], pr["b"],
                        restart=20, maxiter=200, tol=1e-10)
            assert r["N"] == n and r["iterations"] == o["iterations"] and r["status"] == o["status"]
            # the ranks sum on one thread, this process on all: the residual agrees to rounding
            assert abs(r["rel_residual_true"] - o["true_res"]) <= 1e-6 * o["true_res"] + 1e-15
