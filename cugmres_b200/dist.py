"""Multi-GPU plumbing for independent solves (torch.distributed, one process per GPU).

A single GMRES solve does not shard in this library (replicas only); a sweep
of independent systems does: each rank takes a disjoint share of the systems,
balanced by work (grid cells), solves it on its own GPU with
cugmres_solve_batch, and the per-system results are gathered on every rank.
There is no collective on the solve path itself; the only communication is
the final gather of small per-system records and the max-over-ranks timing.
The functions take the solve routine as an argument so the host logic can be
exercised with gloo ranks on CPU.
"""
import numpy as np


def shard_systems(sizes, rank, world):
    """Indices of the systems rank `rank` solves: greedy longest-processing-time
    assignment on N^2 (largest first, to the least loaded rank), deterministic
    on every rank."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]) ** 2, i))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += int(sizes[i]) ** 2
        if r == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (works with nccl and gloo)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_records(records):
    """All-gather a list of per-system dicts (small, pickled) to every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(records)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(records))
    merged = []
    for part in out:
        merged.extend(part)
    return sorted(merged, key=lambda r: r["index"])


def sweep_stats(records, wall_s):
    """solves/s over the whole job and latency percentiles of the systems."""
    lat = np.array([r["seconds"] for r in records], dtype=np.float64)
    conv = sum(1 for r in records if r["status"] == 0)
    return {"systems": len(records), "converged": conv, "wall_s": wall_s,
            "solves_per_s": len(records) / wall_s if wall_s > 0 else None,
            "converged_per_s": conv / wall_s if wall_s > 0 else None,
            "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "iterations_total": int(sum(r["iterations"] for r in records))}


def run_sweep(systems, rank, world, solve_fn, timer=None, device=None):
    """Solve this rank's share with solve_fn(list_of_systems) -> list of info
    dicts, gather every record, return (records, stats).  `timer` returns
    seconds for the local share (default: the duration of the synchronous
    solve_fn call); the job time is the max over ranks (all-reduce on
    `device`: the rank's GPU under NCCL, None for gloo)."""
    import time
    sizes = [int(s["N"]) if "N" in s else s["g_block"].shape[0] for s in systems]
    mine = shard_systems(sizes, rank, world)
    t0 = time.perf_counter()
    infos = solve_fn([systems[i] for i in mine]) if mine else []
    local = timer() if timer else time.perf_counter() - t0
    recs = [dict(index=i, N=sizes[i], **{k: v for k, v in info.items() if k in
                                           ("status", "iterations", "cycles", "seconds", "rel_residual_true")})
            for i, info in zip(mine, infos)]
    records = gather_records(recs)
    job = max_over_ranks(local, device=device)
    return records, sweep_stats(records, job)
