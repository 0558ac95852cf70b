"""Benchmark: GMRES solve of the 1024x1024 Helmholtz GFIEM system (restart 100, tol 1e-10).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--N 1024] [--eps 4] [--restart 100] [--tol 1e-10] [--max-iter 1000]
                    [--precision fp64|mixed]

One step = one GMRES solve of A x = b (x0 = 0) on a synthetic seeded system
with the configuration's shape, sizes and value distribution (no dataset is
involved), stopped at ||b - A x|| / ||b|| <= tol or after --max-iter Arnoldi
steps, whichever comes first.  On the default system (eps_r = 4 scatterer of
about 38 wavelengths) GMRES(100) stagnates near 1e-2, so the step budget ends
the solve: the value is then the time of a budget-capped solve and the JSON
line says so ("solve.converged": false) together with the residual reached.
The value is device time per solve, measured with CUDA events on the solver's
stream, max over ranks; for N > 1 every rank solves its own replica and
value = max rank time / solves of all ranks (replicas only: a single solve
does not shard).

Extra keys: roofline of the dominant phase (algorithmic bytes / live CUDA-event
time vs the measured HBM copy bandwidth in MEASURED_PEAKS.json), e2e (the same
solve through the public API from pinned host buffers, H2D/D2H inside the
timed region), the CPU oracle timed on a bounded sample (rank 0, N = 1), clocks
sampled with nvidia-smi during the timed region.

--impl reference: the reference's CPU GMRES (the oracle's C restatement of
FFT_GMRES_with_MKL generalised to restarts; MKL is absent) on every host
thread, rank 0 only.  It loads nothing of this library: the system is built by
oracle/problems.py with the oracle's own Green's block.  Each timed step is
one whole restart cycle (restart Arnoldi steps, the true residual and the
update); the value scales the mean cycle time by the cycles of the same
budget-capped solve (max_iter / restart).  Warm-up steps run a 5-step sample.

--profile-case: a fixed launch sequence for profiler captures (no timing, no
JSON): three FP64 and three FP32 matvecs of the 1024^2 system, then one solve of
exactly --case-steps Arnoldi steps (tolerance 1e-14, so it never stops early) in
cycles of min(--restart, --case-steps) steps.  With --ortho dcgs2 every step is
[k_rows_forward, k_cols_convolve, k_rows_inverse, k_dots2, k_dcgs2_step, k_axpy2],
so `ncu -k regex:k_dots2 -s 30 -c 1` picks the dot pass of step 30; with the
default s-step scheme a 24-step delayed-CGS2 run gives the shifts first, then
every cycle runs s-step blocks (--sstep), whose passes are k_ss_dots and
k_ss_update.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-10 residual per 1024² solve: learned+mixed vs plain FP64; matvec GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--N", type=int, default=1024)
    ap.add_argument("--eps", type=float, default=4.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--max-iter", type=int, default=1000)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--ortho", default="sstep", choices=["sstep", "dcgs2", "cgs2"],
                    help="Arnoldi scheme of the timed solve (s-step blocks, shifts from a short delayed-CGS2 run)")
    ap.add_argument("--sstep", type=int, default=4, help="steps per s-step block")
    ap.add_argument("--inner-tol", type=float, default=1e-5, help="mixed: a complex64 cycle ends when its estimate fell by this")
    ap.add_argument("--profile-case", action="store_true", help="fixed launch sequence for profiler captures")
    ap.add_argument("--case-steps", type=int, default=60)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the mixed-precision and 256^2 side measurements")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner side measurement")
    ap.add_argument("--learned-steps", type=int, default=1500)
    ap.add_argument("--sweep", type=int, default=64, help="also solve a sweep of this many systems (config 4; 0: none)")
    ap.add_argument("--sweep-max-iter", type=int, default=2000)
    ap.add_argument("--sweep-restart", type=int, default=500,
                    help="restart length of the sweep (64 systems, 2000 steps: 200 -> 14 converged in 6 s, "
                         "500 -> 24 in 8.5 s, mixed precision)")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=5.0):
        """Block until the sampler printed its first line, so that nvidia-smi's
        start-up (NVML initialisation) lies before the timed region."""
        t_end = time.perf_counter() + timeout
        while self.proc is not None and not self.lines and time.perf_counter() < t_end:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def make_problem(args):
    from cugmres_b200 import problems as P
    return P.helmholtz(args.N, args.eps, seed=args.seed)


def workload(args):
    return {"workload": f"helmholtz-gfiem {args.N}x{args.N} eps_r={args.eps:g} seed={args.seed} "
                        f"restart={args.restart} tol={args.tol:g} max_iter={args.max_iter} x0=0 "
                        f"precision={args.precision} ortho={args.ortho}"
                        + (f" sstep={args.sstep}" if args.ortho == "sstep" else ""),
            "ortho": args.ortho, "sstep": args.sstep if args.ortho == "sstep" else None,
            "max_iter": args.max_iter,
            "N": args.N, "unknowns": args.N * args.N, "eps_r": args.eps, "lambda_over_h": 20,
            "restart": args.restart, "tol": args.tol, "precision": args.precision,
            "l2": "inputs larger than L2 (basis of restart+1 vectors of N^2 complex)"}


def oracle_system(args):
    """The benchmark system built by the oracle alone (no libcugmres load)."""
    from oracle import oracle as O
    from oracle import problems as OP
    O.build()
    pr = OP.helmholtz(args.N, args.eps, seed=args.seed)
    gh = O.spectrum(pr["g_block"], OP.embedding(args.N))
    return O, pr, gh


def cycles_per_solve(args):
    """Restart cycles of the budget-capped solve (every cycle runs `restart` steps)."""
    return max(1, -(-args.max_iter // args.restart))


def oracle_cycle(O, pr, gh, args, steps=None):
    """One GMRES(restart) cycle of the oracle in FP64 (or `steps` Arnoldi steps):
    the true residual, the Arnoldi steps with modified Gram-Schmidt, the
    least-squares solve and the update.  Returns seconds."""
    c = pr["chi"] * pr["chi_scale"]
    s = steps or args.restart
    t0 = time.perf_counter()
    out = O.gmres(gh, c, pr["b"], restart=args.restart, maxiter=s, tol=0.0)
    dt = time.perf_counter() - t0
    assert out["iterations"] == s, out["iterations"]
    return dt


def cpu_baseline(args):
    """The oracle (plain-C restatement of the reference's CPU GMRES, MKL absent)
    on every host thread: one whole FP64 GMRES(restart) cycle of the same
    system, scaled by the cycles of the budget-capped solve; next to it the
    reference's own algorithm (FFT_GMRES_with_MKL restated: complex64, no
    restart, modified Gram-Schmidt, explicit Givens products and LU) on one
    core, as the reference's makefile links MKL sequential, timed over its
    first 10 Arnoldi steps."""
    O, pr, gh = oracle_system(args)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    oracle_cycle(O, pr, gh, args, steps=5)  # thread pool and page warm-up
    dt = oracle_cycle(O, pr, gh, args)
    cyc = cycles_per_solve(args)
    out = {"value": dt * cyc, "unit": "s", "cores": threads, "kind": "port",
           "sample": f"one whole FP64 GMRES({args.restart}) cycle of the same {args.N}x{args.N} system "
                     f"({args.restart} Arnoldi steps, true residual, update) in {dt:.2f} s on {threads} threads, "
                     f"x {cyc} cycles of the capped solve"}
    O.set_threads(1)
    s10 = 10
    g64 = gh.astype(np.complex64)
    t0 = time.perf_counter()
    O.gmres_reference(g64, pr["chi"] * pr["chi_scale"], pr["b"], np.zeros_like(pr["b"]), s10, 0.0,
                      precision="c64")
    d1 = time.perf_counter() - t0
    O.set_threads(threads)
    out["reference_1core_c64"] = {
        "value": d1 / s10, "unit": "s per Arnoldi step", "cores": 1, "kind": "port",
        "sample": f"first {s10} steps of FFT_GMRES_with_MKL restated (complex64, unrestarted, MGS) on the "
                  f"{args.N}x{args.N} system, one thread, {d1:.2f} s"}
    return out


def timed_solves(s, b, kw, steps, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    infos = []
    for _ in range(steps):
        x, info = s.solve(b, **kw)
        infos.append(info)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, infos[-1], x


def rel_err(x, ref):
    """||x - ref|| / ||ref|| (x, ref: torch tensors or arrays; None when ref is None)."""
    if ref is None:
        return None
    import torch
    x = torch.as_tensor(x).cpu().numpy().ravel()
    ref = torch.as_tensor(ref).cpu().numpy().ravel()
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


def tight_reference(s, b, restart=2500, max_iter=5000):
    """FP64 GMRES solve tightened to 1e-13, the reference the time-to-tol
    results are compared with; None if it does not get there."""
    x, info = s.solve(b, restart=restart, max_iter=max_iter, tol=1e-13, precision="fp64")
    return x if info["status"] == 0 else None


def side_measurements(args, stream):
    """Mixed precision on the same capped solve; time-to-1e-10 where GMRES
    converges: the 256^2 and 512^2 systems of the same construction
    (unrestarted, by delayed CGS2 in FP64 and mixed precision, and by s-step
    blocks of 4 in FP64; mixed = complex64 cycles that end when their estimate
    fell by 1e-7, FP64 refinement); the config-3 grid (2048^2, eps_r = 12.25, restart
    50) within a budget of 1000 steps, FP64 and mixed."""
    import torch
    import cugmres_b200 as cg
    from cugmres_b200 import problems as P
    out = {}
    pr = make_problem(args)
    s = cg.Solver(torch.cuda.current_device())
    s.set_stream(stream.cuda_stream)
    s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    b = torch.from_numpy(pr["b"]).cuda()
    kw = dict(restart=args.restart, max_iter=args.max_iter, tol=args.tol, precision="mixed", inner_tol=args.inner_tol,
              ortho=args.ortho, sstep=args.sstep)
    s.solve(b, **kw)
    ms, info, _ = timed_solves(s, b, kw, max(1, args.steps), stream)
    out["mixed_capped_solve"] = {"s": ms / 1e3, "steps": info["iterations"], "rel_residual_true": info["rel_residual_true"],
                                 "ms_per_step": ms / max(1, info["iterations"])}
    # the same capped solve with the other Arnoldi schemes: delayed CGS2 (two passes over the
    # basis per step) and s-step blocks of 8
    for prec in ("fp64", "mixed"):
        for name, extra in (("dcgs2", dict(ortho="dcgs2")), ("sstep8", dict(ortho="sstep", sstep=8))):
            kws = dict(restart=args.restart, max_iter=args.max_iter, tol=args.tol, precision=prec,
                       inner_tol=args.inner_tol, **extra)
            s.solve(b, **kws)
            ms, info, _ = timed_solves(s, b, kws, max(1, args.steps), stream)
            out[f"{name}_{prec}_capped_solve"] = {"s": ms / 1e3, "steps": info["iterations"],
                                                 "rel_residual_true": info["rel_residual_true"],
                                                 "ms_per_step": ms / max(1, info["iterations"])}
    s.close()
    for N, R, reps in ((256, 2500, 1), (512, 4400, 0)):
        prn = P.helmholtz(N, args.eps, seed=args.seed)
        s = cg.Solver(torch.cuda.current_device())
        s.set_stream(stream.cuda_stream)
        s.set_operator(prn["g_block"], prn["chi"], prn["chi_scale"])
        bn = torch.from_numpy(prn["b"]).cuda()
        xref = tight_reference(s, bn, restart=R, max_iter=2 * R)
        # delayed CGS2 in FP64 and mixed precision, and s-step blocks of 4 in FP64
        # (shifts refreshed every 100 steps of the long cycle)
        for name, prec, extra in (("fp64", "fp64", {}), ("mixed", "mixed", {}),
                                  ("sstep_fp64", "fp64", dict(ortho="sstep", sstep=4))):
            kwn = dict(restart=R, max_iter=3 * R, tol=args.tol, precision=prec, inner_tol=1e-7, **extra)
            for _ in range(reps):  # warm-up solve (the 512^2 ones are timed cold: graphs are built in their first cycle)
                s.solve(bn, **kwn)
            ms, info, x = timed_solves(s, bn, kwn, 1, stream)
            out[f"time_to_tol_{N}_unrestarted_{name}"] = {
                "s": ms / 1e3, "steps": info["iterations"], "cycles": info["cycles"], "status": info["status_text"],
                "rel_residual_true": info["rel_residual_true"], "err_vs_fp64_tol1e-13": rel_err(x, xref)}
        s.close()
    pr3 = P.helmholtz(2048, 12.25, seed=args.seed)
    s = cg.Solver(torch.cuda.current_device())
    s.set_stream(stream.cuda_stream)
    s.set_operator(pr3["g_block"], pr3["chi"], pr3["chi_scale"])
    b3 = torch.from_numpy(pr3["b"]).cuda()
    row = {}
    for prec in ("fp64", "mixed"):
        kw3 = dict(restart=50, max_iter=1000, tol=args.tol, precision=prec, inner_tol=1e-5)
        ms, info, _ = timed_solves(s, b3, kw3, 1, stream)
        row[prec] = {"s": ms / 1e3, "steps": info["iterations"], "status": info["status_text"],
                     "rel_residual_true": info["rel_residual_true"]}
    row["note"] = ("2048x2048, eps_r = 12.25, GMRES-IR with complex64 cycles of 50 steps; 1e-10 is not reached "
                   "within the 1000-step budget, so no error against a 1e-13 solve exists")
    out["config3_2048_restart50_budget1000"] = row
    s.close()
    return out


def learned_side(args, stream):
    """The learned+mixed arm: a spectral-convolution network trained here on
    the solver's own operators (64^2 designs, eps_r ~ U(2, 6), residual loss,
    not timed) as initial guess and flexible right preconditioner of the
    mixed-precision solve, on the same capped 1024^2 solve and on a 256^2
    time-to-tol solve, next to plain FP64 on the same systems."""
    import torch
    import cugmres_b200 as cg
    from cugmres_b200 import learned as Lr
    from cugmres_b200 import problems as P
    out = {}
    t0 = time.perf_counter()
    ds = Lr.DesignSet(64, 64, seed=500, eps_range=(2.0, 6.0))
    net = Lr.FNO(torch.cuda.current_device(), seed=1)
    hist = Lr.train_residual(net, ds, steps=args.learned_steps, batch=16, lr=1e-3)
    ds.close()
    out["training"] = {"designs": 64, "grid": 64, "steps": args.learned_steps, "seconds": time.perf_counter() - t0,
                       "final_residual_loss": float(np.mean(hist[-100:]))}
    for N, restart, maxit in ((args.N, args.restart, args.max_iter), (256, 2500, 2500)):
        pr = P.helmholtz(N, args.eps, seed=args.seed)
        s = cg.Solver(torch.cuda.current_device())
        s.set_stream(stream.cuda_stream)
        s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
        s.set_preconditioner(net, pr["k0"] * pr["h"])
        b = torch.from_numpy(pr["b"]).cuda()
        # the capped 1024^2 solve has no converged reference (GMRES stagnates near 1e-2)
        xref = tight_reference(s, b) if N <= 256 else None
        row = {}
        for name, kw in (("plain_fp64", dict(precision="fp64")),
                         ("learned_mixed", dict(precision="mixed", preconditioner="learned", learned_x0=True,
                                                inner_tol=1e-6))):
            kw.update(restart=restart, max_iter=maxit, tol=args.tol)
            s.solve(b, **kw)
            ms, info, x = timed_solves(s, b, kw, 1, stream)
            row[name] = {"s": ms / 1e3, "steps": info["iterations"], "status": info["status_text"],
                         "rel_residual_true": info["rel_residual_true"],
                         "preconditioned_cycles": info["preconditioned_cycles"], "x0_learned": info["x0_learned"],
                         "err_vs_fp64_tol1e-13": rel_err(x, xref)}
        s.set_preconditioner(None)
        s.close()
        out[f"{N}x{N}_restart{restart}_max_iter{maxit}"] = row
    net.close()
    return out


def sweep_side(args, rank, world, device, precision="mixed"):
    """Config 4: independent systems with sides drawn from {96,...,512}, lambda/h
    ~ U(15, 30), eps_r ~ U(2, 12), one design seed each, solved in lockstep
    buckets (cugmres_solve_buckets: one launch per kernel per Arnoldi step for
    all systems of a bucket, one CUDA-graph replay per restart cycle, operators
    built on the GPU), GMRES(--sweep-restart) to 1e-10 within --sweep-max-iter steps, in
    mixed precision (complex64 cycles that end when their estimate fell by 1e-7,
    FP64 residual and update) or FP64.  With
    N ranks the systems are sharded largest-first over the ranks (no collective
    on the solve path); the job time is the maximum over ranks of each rank's
    synchronous sweep call (it returns when its GPU work is done), and the
    per-system records are gathered to every rank."""
    import cugmres_b200 as cg
    from cugmres_b200 import dist as D
    from cugmres_b200 import problems as P
    systems = P.sweep(nsys=args.sweep, seed=0, with_green=False)
    kw = dict(device=device, mode="buckets", restart=args.sweep_restart, tol=args.tol, precision=precision,
              inner_tol=1e-7)
    # untimed: one short solve per grid side of this rank's share, so every
    # embedding size is autotuned before the clock starts
    mine = D.shard_systems([s["N"] for s in systems], rank, world)
    warm, seen = [], set()
    for i in mine:
        if systems[i]["N"] not in seen:
            seen.add(systems[i]["N"])
            warm.append(systems[i])
    if warm:
        cg.solve_batch(warm, max_iter=20, **kw)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()

    def solve_fn(lst):
        return cg.solve_batch(lst, max_iter=args.sweep_max_iter, **kw)[1]

    records, stats = D.run_sweep(systems, rank, world, solve_fn, device=f"cuda:{device}")
    stats.update({"gpus": world, "matvecs_per_s": float(sum(r["iterations"] + r["cycles"] for r in records) /
                                                        stats["wall_s"]) if stats["wall_s"] else None,
                  "arnoldi_steps": int(sum(r["iterations"] for r in records)),
                  "by_side": {str(N): {"systems": sum(1 for r in records if r["N"] == N),
                                       "converged": sum(1 for r in records if r["N"] == N and r["status"] == 0)}
                              for N in sorted({r["N"] for r in records})},
                  "precision": precision,
                  "note": (f"GMRES({args.sweep_restart}), tol {args.tol:g}, at most {args.sweep_max_iter} steps per "
                           "system; "
                           "latency = from the start of the system's bucket (set-up included) to the cycle "
                           "at which it finished")})
    return stats


def run_reference(args, rank, world):
    """The reference's CPU GMRES (oracle port: MKL absent) on the host cores,
    rank 0 only; nothing of this library is loaded."""
    if rank != 0:
        return
    O, pr, gh = oracle_system(args)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    for _ in range(args.warmup):
        oracle_cycle(O, pr, gh, args, steps=5)
    times = [oracle_cycle(O, pr, gh, args) for _ in range(args.steps)]
    cyc = cycles_per_solve(args)
    per_cycle = float(np.mean(times))
    v = per_cycle * cyc
    sample = (f"each timed step is one whole FP64 GMRES({args.restart}) cycle of the oracle (modified "
              f"Gram-Schmidt, {threads} threads) on the same {args.N}x{args.N} system, mean {per_cycle:.2f} s; "
              f"value = cycle time x {cyc} cycles of the budget-capped solve; warm-up steps run 5 Arnoldi steps")
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_cycle * 1e3,
            "ms_per_step_unit": "ms per restart cycle (the timed sample)", "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": workload(args),
            "cpu_baseline": {"kind": "port", "cores": threads, "sample": sample, "value": v, "unit": "s"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_case(args):
    """Fixed launch sequence for profiler captures (see the module docstring)."""
    import cugmres_b200 as cg
    from cugmres_b200 import problems as P
    pr = P.helmholtz(args.N, args.eps, seed=args.seed)
    s = cg.Solver(0)
    s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = np.random.default_rng(0).standard_normal((args.N, args.N)) + 0j
    for _ in range(3):
        s.matvec(x)
    x32 = x.astype(np.complex64)
    for _ in range(3):
        s.matvec(x32, precision="fp32")
    _, info = s.solve(pr["b"], restart=min(args.restart, args.case_steps), max_iter=args.case_steps, tol=1e-14,
                      precision=args.precision, ortho=args.ortho, sstep=args.sstep)
    s.close()
    print("ok", info["iterations"], info["status_text"], flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.profile_case:
        return profile_case(args)

    import torch
    import torch.distributed as dist
    import cugmres_b200 as cg

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    pr = make_problem(args)
    stream = torch.cuda.current_stream()
    s = cg.Solver(local)
    s.set_stream(stream.cuda_stream)
    s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    b_dev = torch.from_numpy(pr["b"]).cuda()
    kw = dict(restart=args.restart, max_iter=args.max_iter, tol=args.tol, precision=args.precision,
              inner_tol=args.inner_tol, ortho=args.ortho, sstep=args.sstep)

    for _ in range(args.warmup):
        x, info = s.solve(b_dev, **kw)
    torch.cuda.synchronize()

    clocks = Clocks(local)
    clocks.start()
    clocks.wait_first()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms_one, last, _ = timed_solves(s, b_dev, kw, args.steps, stream)
    if world > 1:
        dist.barrier()
    ms_total = ms_one * args.steps
    clk = clocks.stop()
    # phase breakdown from one more solve with CUDA events between kernel groups (not timed;
    # events disable the graph replay)
    s.profile(True)
    s.solve(b_dev, **kw)
    torch.cuda.synchronize()
    prof = s.profile_read()
    s.profile(False)

    # end to end through the public API from pinned host memory
    b_host = torch.from_numpy(pr["b"]).pin_memory()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        xh, info_h = s.solve(b_host.numpy(), **kw)
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_wall = (time.perf_counter() - t0) / args.steps

    t = torch.tensor([ms_total], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps
    value = ms_per_step / 1e3 / world  # seconds per solve over all ranks' solves

    hbm, peak_kind = peaks()
    phases = {k: v for k, v in prof.items() if v["ms"] > 0}
    dom = max(phases.items(), key=lambda kv: kv[1]["ms"])
    tot_ms = sum(v["ms"] for v in phases.values())
    # DRAM traffic per launch of the dominant kernel is not measurable without a profiler: it is taken
    # from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the launch at step k = 30
    # (delayed CGS2) or of the block at k = 48 (s-step) of this 1024^2 FP64 solve (bench.py
    # --profile-case), as a ratio to that launch's algorithmic bytes, applied to this run's mean
    # algorithmic bytes per launch; "traffic_source" says so
    if args.ortho == "sstep":
        # k_ss_dots / k_ss_update of the block at k = 48 of a 1024^2 FP64 GMRES(100) s-step cycle (S = 4):
        # 53 vectors read (889.19 MB); the update also writes the 4 block vectors (956.30 MB in all),
        # most of which are still in L2 when the kernel ends
        ncu_ratio = {"dots": (889.260 + 4.386) / 889.192, "axpy": (889.234 + 55.452) / 956.301}
    else:
        ncu_ratio = {"dots": (536.904 + 4.625) / 536.871, "axpy": (536.961 + 8.369) / 570.425}
    # the three FFT passes of one FP64 matvec at 1024^2 (the same capture's DRAM read + write of
    # k_rows_forward, k_cols_convolve_pipe, k_rows_inverse) against the 16 n e model (268.44 MB):
    # replayed with flushed caches, each pass reads its inputs from DRAM while the intermediate
    # it writes is still in L2 when it ends
    ncu_ratio["matvec"] = (25.189 + 0.139 + 50.408 + 0.139 + 50.363 + 0.473) / 268.435
    launches = max(1, dom[1].get("launches", 0))
    alg_per_launch = dom[1].get("bytes", 0.0) / launches
    if dom[0] == "matvec":
        # per operator application (its three FFT passes): a profile interval of an s-step block
        # holds S of them, so the phase's mean interval is not one application
        alg_per_launch = 16.0 * args.N * args.N * (16 if args.precision == "fp64" else 8)
    traffic = ncu_ratio[dom[0]] * alg_per_launch if dom[0] in ncu_ratio and alg_per_launch > 0 else None
    roof = {"bound": "hbm", "kernel": dom[0], "achieved": round(dom[1]["gbs"], 1), "peak": hbm, "unit": "GB/s",
            "frac": round(dom[1]["gbs"] / hbm, 4), "peak_kind": peak_kind,
            "traffic": round(traffic) if traffic else None,
            "traffic_unit": "bytes/matvec (three FFT launches)" if dom[0] == "matvec" else "bytes/launch",
            "traffic_source": ("ncu capture of the same kernels of this solve (matvec: its three FFT passes; "
                               "delayed CGS2: step 30; s-step: the block at k = 48), their DRAM bytes / "
                               "algorithmic bytes ratio applied to this run's mean launch"),
            "algorithmic_bytes_per_launch": round(alg_per_launch),
            "phases": {k: {"share": round(v["ms"] / tot_ms, 4), "gbs": round(v["gbs"], 1),
                           "ms": round(v["ms"], 3)} for k, v in phases.items()}}
    mv = prof.get("matvec", {})
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128" if args.precision == "fp64" else "c64/c128",
            "data": "synthetic", "config": workload(args),
            "solve": {"converged": last["status"] == 0, "status": last["status_text"], "steps": last["iterations"],
                      "cycles": last["cycles"], "rel_residual_true": last["rel_residual_true"],
                      "ms_per_step": ms_per_step / max(1, last["iterations"]),
                      "note": ("tol reached" if last["status"] == 0 else
                               f"tol {args.tol:g} not reached within {args.max_iter} Arnoldi steps: "
                               "value is the time of the budget-capped solve")},
            "matvec_shapes": {"fp64": list(s.matvec_shapes("fp64")), "fp32": list(s.matvec_shapes("fp32"))},
            "matvec_gbs": round(mv.get("gbs", 0.0), 1),
            "roofline": roof,
            "e2e": {"value": e2e_wall, "unit": "s", "h2d_bytes_per_step": int(pr["b"].nbytes),
                    "d2h_bytes_per_step": int(pr["b"].nbytes)},
            "gpu_launches": None, "clocks": clk}
    # our kernels per solve, counted from the enqueued sequence (launches after the device stops a
    # cycle return at once): the norm of b, the first residual (3 passes) and cycle set-up; per
    # delayed-CGS2 cycle 6 per step (3 matvec passes, dots, step, axpy) for restart+1 steps, then
    # back-solve, update, 3 residual passes and the cycle set-up; an s-step cycle instead runs q_0's
    # normalisation, per block of S steps 2 S + 1 matvec passes (the inverse row pass of each chained
    # matvec but the last also runs the next forward row pass), 2 x (dots with the Cholesky in their
    # last block, update) and the Hessenberg/Givens kernel, then the same 6
    per_dcgs2 = 6 * (args.restart + 1) + 6
    per_ss = 1 + -(-args.restart // args.sstep) * (2 * args.sstep + 6) + 6
    cyc = last["cycles"]
    per_solve = 5 + (per_dcgs2 + (cyc - 1) * per_ss if args.ortho == "sstep" else cyc * per_dcgs2)
    line["gpu_launches"] = int(args.steps * per_solve)
    if rank == 0 and world == 1 and not args.no_extras:
        line["side"] = side_measurements(args, stream)
        if not args.no_learned:
            line["side"]["learned"] = learned_side(args, stream)
    if args.sweep > 0:
        line.setdefault("side", {})["sweep"] = sweep_side(args, rank, world, local, "mixed")
        line["side"]["sweep_fp64"] = sweep_side(args, rank, world, local, "fp64")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
