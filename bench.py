#!/usr/bin/env python
"""Benchmark: solves/s of the HODLR direct solve on B200.

Workload (default): N = 262144 unknowns, dense leaves of 512 rows (512 leaves,
9 levels), rank 64 at every level, 16 right-hand sides; seeded synthetic
system (leaf blocks G/sqrt(512) + 2I, U/V iid Gaussian rescaled so every
off-diagonal block has spectral norm 0.5, b iid N(0,1)), generated on the
device.  One step = one solve of that system with its whole RHS block:

  value     mixed precision: FP32 leaf LU, FP32 reduce/broadcast, FP64 node
            LU, FP64 HODLR-matvec residual and FP64 refinement sweeps until
            max_j ||b_j - A x_j|| / ||b_j|| <= 1e-12 (factor + refinement
            inside every step)
  fp64_gpu  the plain FP64 path (the fused factor+solve of the reference's
            bfs_solve), same system, timed the same way
  e2e       `value`'s solve through the public API with the system in pinned
            host memory: one hodlr_solve_refined_host call per step (H2D of
            D, U, V, b, with V's copy under the leaf factorization, the
            refined solve, D2H of x)
  --impl reference: the CPU oracle (a restatement of the reference's
            Legion+LAPACK path with OpenBLAS, all host threads) on the same
            workload, printed as the reference arm.

Inputs are ~3.5 GB, far above the 126 MB L2, so no explicit flush is needed.
Multi-GPU (torchrun): every rank solves its own system (replicas, weak
scaling, no collective on the data path); value = total solves / max time.
"""
from __future__ import annotations

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

CONFIGS = {
    "n262144": dict(N=262144, leaf=512, rank=64, nrhs=16),   # the metric's system
    "n65536": dict(N=65536, leaf=512, rank=50, nrhs=8),
    "n4096": dict(N=4096, leaf=256, rank=30, nrhs=1),
    "n1048576": dict(N=1048576, leaf=512, rank=100, nrhs=32),
}
METRIC = "solves/s at N=2^18,r=64: mixed+batched vs plain FP64 GPU @relres<=1e-12"
# batched workload: 64 independent systems, N log-uniform in [8192, 131072],
# leaf size from {256, 512, 1024}, rank uniform in [16, 96], 1..32 RHS
BATCH = dict(count=64, n_lo=8192, n_hi=131072, leaves=(256, 512, 1024), rank=(16, 96),
             nrhs=(1, 32))
BATCH_METRIC = "systems solved/s: 64 uneven HODLR systems, batched mixed @relres<=1e-12"
TOL = 1e-12


# ---------------------------------------------------------------------------
# algorithmic work of one fused solve (per phase), from the tree
# ---------------------------------------------------------------------------

def work_model(tree: np.ndarray, m: int):
    """Flops and compulsory bytes (FP64 words x 8) of one fused factor+solve."""
    nrow, ncol, rb, cb, lc, rc, par, dep, vnc, leaf = (tree[:, i] for i in range(10))
    w = dict(getrf=0.0, getrs=0.0, reduce=0.0, node=0.0, broadcast=0.0)
    for i in range(tree.shape[0]):
        if leaf[i]:
            n = float(nrow[i])
            c = float(cb[i] + ncol[i])
            w["getrf"] += 2.0 / 3.0 * n ** 3
            w["getrs"] += 2.0 * n * n * c
            continue
        a, b = lc[i], rc[i]
        cw = float(cb[a])
        r0, r1 = float(ncol[a]), float(ncol[b])
        for ch in (a, b):
            w["reduce"] += 2.0 * nrow[ch] * vnc[ch] * (cb[ch] + ncol[ch])
            w["broadcast"] += 2.0 * nrow[ch] * ncol[ch] * cw
        w["node"] += 2 * r0 * r1 * r0 + 2.0 / 3.0 * r0 ** 3 + 2 * r0 * r0 * cw + 4 * r0 * r1 * cw
    return w


def phase_bytes(tree: np.ndarray, m: int, word: int):
    """Compulsory bytes per phase of one fused solve in `word`-byte arithmetic."""
    nrow, ncol, rb, cb, lc, rc, par, dep, vnc, leaf = (tree[:, i] for i in range(10))
    b = dict(getrf=0.0, getrs=0.0, reduce=0.0, node=0.0, broadcast=0.0)
    for i in range(tree.shape[0]):
        if leaf[i]:
            n = float(nrow[i])
            c = float(cb[i] + ncol[i])
            b["getrf"] += 2 * n * n * word          # read D, write LU
            b["getrs"] += (n * n + 2 * n * c) * word  # read LU, read+write X
            continue
        a, bb = lc[i], rc[i]
        cw = float(cb[a])
        for ch in (a, bb):
            b["reduce"] += nrow[ch] * (vnc[ch] + cb[ch] + ncol[ch]) * word
            b["broadcast"] += nrow[ch] * (ncol[ch] + 2 * cw) * word
    return b


def leaf_update_bytes(tree: np.ndarray, word: int, nb: int = 64, ob: int = 0) -> float:
    """Algorithmic bytes of all leaf trailing-update GEMMs (C -= A B) of one
    factor pass of the two-level blocked LU (outer blocks of `ob` columns,
    panels of `nb`; ob <= nb is one level): per update item, C read and
    written, A and B read once.  The items are those the library builds:
    inside each block (rows below the panel x the block's columns right of
    it), on the block rows (x the columns right of the block | X) when those
    are solved panel by panel (ob > 128), and the depth-ob trailing update
    (rows below the block x the same columns).  With nb < ob <= 128 the block
    rows are solved by one product with the block's triangular inverse (a
    solve, not an update)."""
    nrow, ncol, rb, cb, lc, rc, par, dep, vnc, leaf = (tree[:, i] for i in range(10))
    ob = ob // nb * nb if ob >= nb else nb
    binv = nb < ob <= 128
    tot = 0.0

    def item(M, N, K):
        return word * (2.0 * M * N + M * K + K * N) if M > 0 and N > 0 and K > 0 else 0.0

    for i in range(tree.shape[0]):
        if not leaf[i]:
            continue
        n = int(nrow[i])
        ncols = int(cb[i] + ncol[i])
        for j0 in range(0, n, ob):
            obe = min(ob, n - j0)
            R = n - j0 - obe + ncols
            for k0 in range(j0, j0 + obe, nb):
                kb = min(nb, n - k0)
                tot += item(n - k0 - kb, j0 + obe - k0 - kb, kb)   # inside the block
                if not binv:
                    tot += item(j0 + obe - k0 - kb, R, kb)         # block rows
            tot += item(n - j0 - obe, R, obe)                      # trailing, depth ob
    return tot


def profile_traffic(path: str):
    """DRAM bytes per launch (read + write) recorded by an ncu capture summary."""
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return dict(hbm=float(p["hbm_gbs"]), bf16=float(p["bf16_tflops"]),
                    sm_mhz=float(p.get("sm_max_mhz", 1965.0)), src="measured")
    return dict(hbm=6650.0, bf16=1590.0, sm_mhz=1965.0, src="fallback")


def simt_peak_tflops(word: int, sm_mhz: float) -> float:
    """Nominal SIMT FMA peak: 148 SMs x (128 FP32 | 64 FP64) FMA/clk x 2."""
    lanes = 128 if word == 4 else 64
    return 148 * lanes * 2 * sm_mhz * 1e6 / 1e12


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_max(x: float, dist=None, device="cuda") -> float:
    """Max of a per-rank scalar over all ranks (the timing rule: the slowest
    rank defines the step time); identity without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ms_max: float, world_size: int) -> float:
    """Whole-job solves/s of `world_size` replicas, each one solve per step."""
    return world_size * 1e3 / ms_max


def make_system(fs, cfg, seed):
    h = fs.HodlrMatrix(cfg["nrhs"], cfg["N"], cfg["rank"], cfg["leaf"]).create_tree()
    h.init_gaussian(seed, 0.5)
    return h


def batch_systems(seed: int, count: int = BATCH["count"]):
    """The batched workload's seeded draw of system shapes."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        N = int(round(np.exp(rng.uniform(np.log(BATCH["n_lo"]), np.log(BATCH["n_hi"])))))
        leaf = int(rng.choice(BATCH["leaves"]))
        rank = int(rng.integers(BATCH["rank"][0], BATCH["rank"][1] + 1))
        nrhs = int(rng.integers(BATCH["nrhs"][0], BATCH["nrhs"][1] + 1))
        out.append(dict(N=N, leaf=leaf, rank=rank, nrhs=nrhs))
    return out


def run_batch(args):
    """Batched workload: every step solves all systems of the draw in one
    merged schedule (SystemBatch, mixed precision + FP64 refinement to
    relres <= 1e-12).  Beside it: the same systems solved one after another
    with the single-system mixed solve, and with the plain FP64 path."""
    import torch
    import fastsolver_b200 as fs
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    cfgs = batch_systems(args.seed)
    hs = [make_system(fs, c, args.seed + 7919 * rank + i) for i, c in enumerate(cfgs)]
    batch = fs.SystemBatch(hs)
    solver = fs.FastSolver()

    # profiling runs launch eagerly on the legacy default stream (no CUDA
    # graphs), so that the profiler sees ordinary kernel launches
    run_stream = None if args.profile_one else stream

    def batch_step():
        return batch.solve_refined(tol=TOL, maxiter=10, stream=run_stream)

    tune_info = None
    if args.schedule:
        for h in hs:
            h.schedule = json.loads(args.schedule)
        batch.close()
        batch = fs.SystemBatch(hs)
    elif not args.no_tune and not args.profile_one:
        best, ms, trials = batch.autotune(tol=TOL, reps=1)
        tune_info = {"schedule": best, "ms": round(ms, 4), "trials": len(trials)}

    if args.profile_one:
        for _ in range(2):
            batch_step()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        batch_step()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(f"profiled one batched solve of {len(hs)} systems", flush=True)
        return

    def timed(fn, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0.record(stream)
        out = [fn() for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        return rank_max(e0.elapsed_time(e1) / steps, dist, "cuda"), out

    for _ in range(args.warmup):
        batch_step()
    clocks = ClockSampler(local)
    clocks.start()
    fs.reset_launch_count()
    ms_batch, outs = timed(batch_step, args.steps)
    launches = fs.launch_count()
    clk = clocks.stop()
    sweeps = [o[0] for o in outs]
    rr_max = max(max(o[1]) for o in outs)
    x_batch = [h.solution(stream=stream) for h in hs]   # outside the timed region

    def seq_mixed():
        return [solver.solve_refined(h, fs.PREC_MIXED, tol=TOL, maxiter=10, stream=stream)
                for h in hs]

    def seq_fp64():
        for h in hs:
            solver.bfs_solve(h, sync=False, stream=stream)

    # the FP64 path with the two-level FP64 leaf LU (the autotuner's choice
    # for that path at N = 262144); the batch's own schedule is unchanged
    for h in hs:
        h.schedule = {"leaf_ob64": 128}

    for _ in range(2):
        seq_mixed()
    ms_seq, _ = timed(seq_mixed, max(1, args.steps // 2))
    for _ in range(2):
        seq_fp64()
    ms_fp64, _ = timed(seq_fp64, max(1, args.steps // 2))
    rr_fp64 = max(h.relres(stream=stream) for h in hs)

    batch.set_profiling(True)
    batch_step()
    ph = batch.phase_times(reset=True)
    batch.set_profiling(False)

    # the oracle (restated reference FP64 walk) on the host cores: systems of
    # the draw one after another, in draw order, until about args.cpu_seconds
    # of CPU time; the batched solutions' forward error against its solutions
    cpu, fwd = None, None
    if not args.no_cpu_baseline and rank == 0:
        from oracle import refcpu as R
        threads = os.cpu_count() or 1
        R.lib().ref_set_blas_threads(1)
        errs, t_cpu, n_cpu = [], 0.0, 0
        for i, h in enumerate(hs):
            if t_cpu > args.cpu_seconds:
                break
            D, U, V, B = h.get_matrix()
            so = R.System(h.tree_nodes(), D, U, V, B)
            t0 = time.perf_counter()
            Xc, _ = R.bfs_solve(so, nthreads=threads)
            t_cpu += time.perf_counter() - t0
            n_cpu += 1
            errs.append(R.rel_error(x_batch[i], Xc[:, : cfgs[i]["nrhs"]]))
        cpu = {"value": n_cpu / t_cpu, "unit": "systems/s", "cores": threads, "kind": "port",
               "sample": f"the first {n_cpu} of the {len(hs)} systems, fused FP64 solves one "
                         "after another (oracle/refcpu.c, OpenBLAS, one OpenMP task per "
                         "leaf/node)"}
        fwd = {"batched_mixed_vs_oracle_max": max(errs), "systems_checked": n_cpu}
    if rank == 0:
        n = len(hs)
        line = {
            "metric": BATCH_METRIC, "value": ws * n * 1e3 / ms_batch, "unit": "systems/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64",
            "data": "synthetic (seeded Gaussian HODLR systems generated on the device)",
            "config": {"workload": f"{n} uneven HODLR systems, batched mixed+refine to "
                                   f"relres<=1e-12", **BATCH,
                       "unknowns": int(sum(c["N"] for c in cfgs)), "seed": args.seed,
                       "parallelism": f"replicas x{ws}",
                       "l2": "inputs tens of GB > L2"},
            "relres_max": rr_max, "refine_sweeps": sweeps,
            "sequential_mixed": {"value": ws * n * 1e3 / ms_seq, "unit": "systems/s",
                                 "ms_per_step": ms_seq},
            "sequential_fp64": {"value": ws * n * 1e3 / ms_fp64, "unit": "systems/s",
                                "ms_per_step": ms_fp64, "relres": rr_fp64},
            "batched_over_sequential_mixed": ms_seq / ms_batch,
            "batched_over_sequential_fp64": ms_fp64 / ms_batch,
            "phases_ms": {k: round(v[0], 4) for k, v in ph.items()},
            "schedule": hs[0].schedule, "autotune": tune_info,
            "gpu_launches": int(launches), "clocks": clk,
            "forward_err": fwd,
            "e2e": None, "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# reference arm: the CPU oracle (restated reference path) on the host cores
# ---------------------------------------------------------------------------

def run_reference(args, cfg):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import refcpu as R
    threads = os.cpu_count() or 1
    s = R.gaussian_system(cfg["N"], cfg["nrhs"], cfg["rank"], cfg["leaf"], seed=args.seed)
    R.lib().ref_set_blas_threads(1)
    for _ in range(args.warmup):
        R.bfs_solve(s, nthreads=threads)
    t0 = time.perf_counter()
    rr = 0.0
    for _ in range(args.steps):
        X, _ = R.bfs_solve(s, nthreads=threads)
    dt = time.perf_counter() - t0
    rr = R.relres(s, X[:, : cfg["nrhs"]])
    v = args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian HODLR system, numpy PCG64)",
        "config": {"workload": f"hodlr_solve N={cfg['N']} leaf={cfg['leaf']} r={cfg['rank']} "
                               f"m={cfg['nrhs']}", **cfg, "relres": rr},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full fused FP64 solves (oracle/refcpu.c: "
                                   "restated task bodies + BFS walk, OpenBLAS dgesv/dgemm, "
                                   "one OpenMP task per leaf/node of a level)"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="n262144", choices=sorted(CONFIGS) + ["batch64"])
    ap.add_argument("--seed", type=int, default=1245667)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-solves", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="CPU time budget of the batched workload's oracle sample")
    ap.add_argument("--cpu-baseline-large", action="store_true",
                    help="run the oracle leg also above N = 2^18 (needs ~40 GB of host "
                         "memory at N = 2^20)")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch schedule (skip the autotuner)")
    ap.add_argument("--schedule", default=None,
                    help="JSON launch schedule for every path (skips the autotuner), e.g. "
                         "'{\"leaf_ob32\": 256}'")
    ap.add_argument("--profile-one", choices=["mixed", "fp64", "batch"], default=None,
                    help="warm up, then run one solve between cudaProfilerStart/Stop and exit "
                         "(for ncu --profile-from-start off); prints no bench line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.config == "batch64":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched workload has "
                              "no reference counterpart (one system per reference run)"}))
            return
        return run_batch(args)
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference(args, cfg)

    import torch
    import fastsolver_b200 as fs

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return rank_max(x, dist, "cuda")

    # a side stream: the solve's replayable segments are captured as CUDA
    # graphs on their first call (the legacy default stream cannot be captured)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    h = make_system(fs, cfg, args.seed + rank)
    tree = h.tree_nodes()
    solver = fs.FastSolver()
    # launch schedules from the autotuner (untimed): one per path, installed
    # before that path's warm-up
    if args.schedule:
        h.schedule = json.loads(args.schedule)
    sched_default = h.schedule
    sched = {"mixed": sched_default, "fp64": sched_default}
    tune_info = None
    if not args.no_tune and not args.profile_one and not args.schedule:
        tune_info = {}
        for name, prec in (("mixed", fs.PREC_MIXED), ("fp64", fs.PREC_FP64)):
            h.schedule = sched_default
            best, ms, trials = h.autotune(prec, tol=TOL, reps=2)
            sched[name] = best
            tune_info[name] = {"schedule": best, "ms": round(ms, 4), "trials": len(trials)}
    h.schedule = sched["mixed"]

    # profiling runs launch eagerly on the legacy default stream (no CUDA
    # graphs), so that the profiler sees ordinary kernel launches
    run_stream = None if args.profile_one else stream

    def mixed_step():
        it, rr = solver.solve_refined(h, fs.PREC_MIXED, tol=TOL, maxiter=10, stream=run_stream)
        return it, rr

    def fp64_step():
        solver.bfs_solve(h, sync=False, stream=run_stream)

    if args.profile_one:
        step = mixed_step if args.profile_one == "mixed" else fp64_step
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        step()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(f"profiled one {args.profile_one} solve of {args.config}", flush=True)
        return

    # ---- warm-up
    for _ in range(args.warmup):
        mixed_step()
    torch.cuda.synchronize()

    # ---- timed: mixed precision (the metric's value)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    fs.reset_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters, rrs = [], []
    e0.record(stream)
    for _ in range(args.steps):
        it, rr = mixed_step()
        iters.append(it)
        rrs.append(rr)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = fs.launch_count()
    clk = clocks.stop()
    ms_mixed = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    barrier()
    x_mixed = h.solution(stream=stream)   # the last timed solve's x (outside the timing)

    # ---- timed: plain FP64 path
    h.schedule = sched["fp64"]
    for _ in range(args.warmup):
        fp64_step()
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        fp64_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_fp64 = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    rr_fp64 = h.relres(stream=stream)
    x_fp64 = h.solution(stream=stream)

    # ---- per-phase device time (separate, event-bracketed passes)
    h.set_profiling(True)
    fp64_step()
    torch.cuda.synchronize()
    ph_fp64 = h.phase_times(reset=True)
    h.schedule = sched["mixed"]
    mixed_step()
    ph_mixed = h.phase_times(reset=True)
    h.set_profiling(False)

    # ---- end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        D, U, V, B = h.get_matrix()
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).pin_memory()  # noqa: E731
        Dp, Up, Vp, Bp = pin(D), pin(U), pin(V), pin(B)
        xout = torch.empty((cfg["nrhs"], cfg["N"]), dtype=torch.float64).pin_memory()
        N = cfg["N"]
        from fastsolver_b200._lib import call
        import ctypes

        it_e, rr_e = ctypes.c_int(), ctypes.c_double()

        def e2e_step():
            # one host-to-host call: D, U, V, b in from pinned memory (V's copy
            # under the leaf factorization), refined solve, x out
            call("hodlr_solve_refined_host", h.handle, Dp.data_ptr(), N, Up.data_ptr(), N,
                 Vp.data_ptr(), N, Bp.data_ptr(), N, xout.data_ptr(), N, fs.PREC_MIXED, TOL, 10,
                 ctypes.byref(it_e), ctypes.byref(rr_e), stream.cuda_stream)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        ksteps = max(2, min(args.steps, 5))
        e0.record(stream)
        for _ in range(ksteps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1) / ksteps)
        h2d = (Dp.numel() + Up.numel() + Vp.numel() + Bp.numel()) * 8
        e2e = {"value": replica_value(ms_e2e, ws), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(xout.numel() * 8), "ms_per_step": ms_e2e,
               "steps": ksteps, "relres": rr_e.value, "refine_sweeps": it_e.value}

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel and of the whole solve
    pk = peaks()
    m = cfg["nrhs"]
    W = work_model(tree, m)
    B4 = phase_bytes(tree, m, 4)
    B8 = phase_bytes(tree, m, 8)
    fp32_peak = simt_peak_tflops(4, pk["sm_mhz"])
    fp64_peak = simt_peak_tflops(8, pk["sm_mhz"])
    # Dominant kernel: the leaf trailing updates A22 -= L21 U12 of the blocked
    # FP32 leaf factorization (tcgen05 split-BF16 GEMM engine), HBM-bound at
    # K = 64.  Algorithmic bytes per launch = read + write of the updated
    # block plus both operands, FP32, averaged over the launches; duration =
    # the CUDA-event time of those launches in one factor pass / launches.
    h.set_profiling(True)
    solver.factor(h, fs.PREC_MIXED, stream=stream)
    ph_f = h.phase_times(reset=True)
    h.set_profiling(False)
    ms_upd, n_upd = ph_f["leaf_update"]
    sm = sched["mixed"]
    nb_used = sm["leaf_nb"] or (64 if int(tree[tree[:, 9] == 1, 0].max()) <= 512 else 32)
    upd_bytes = leaf_update_bytes(tree, 4, nb_used, sm["leaf_ob32"])
    per_launch_ms = ms_upd / max(n_upd, 1)
    bytes_per_launch = upd_bytes / max(n_upd, 1)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    # DRAM bytes per launch from the ncu capture of this workload (recorded
    # for the 262144-row system only; none for the other configs)
    traffic = (profile_traffic(os.path.join(ROOT, "profiles", "leaf_update_gemm_n262144.md"))
               if args.config == "n262144" else None)
    roofline = {"bound": "hbm", "kernel": "tc_gemm_persistent<128,false,float,true> (leaf trailing update)",
                "achieved": achieved, "peak": pk["hbm"], "unit": "GB/s",
                "frac": achieved / pk["hbm"], "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "ms_per_launch": per_launch_ms, "launches": n_upd,
                "peak_note": "measured HBM copy bandwidth of this pool's B200s"
                             if pk["src"] == "measured" else "fallback 6650 GB/s"}

    def solve_frac(ms, word, peak_tf, passes=1):
        """Roofline time of one fused solve / measured: every phase at the slower
        of its flops (x passes: 3 for split-BF16) and its compulsory bytes."""
        Bx = B4 if word == 4 else B8
        t = 0.0
        for k in ("getrf", "getrs", "reduce", "broadcast"):
            t += max(passes * W[k] / (peak_tf * 1e12), Bx[k] / (pk["hbm"] * 1e9))
        t += W["node"] / (fp64_peak * 1e12)
        return t * 1e3 / ms

    total_flops = sum(W.values())

    def rel(x, ref):
        return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))

    # forward error (the reference's Err formula, direct_solve.cc:216-225):
    # the mixed solution against the FP64 GPU solution always, and both
    # against the oracle's FP64 solve of the same system with the CPU leg
    fwd = {"mixed_vs_fp64_gpu": rel(x_mixed, x_fp64)}
    relres_oracle = None
    cpu = None
    # the oracle holds the system and its working arrays in host memory
    # (~40 GB at N = 2^20), so by default its leg runs up to N = 2^18
    cpu_leg = (not args.no_cpu_baseline and ws == 1
               and (cfg["N"] <= 262144 or args.cpu_baseline_large))
    if cpu_leg:
        from oracle import refcpu as R
        D, U, V, B = h.get_matrix()
        s = R.System(tree, D, U, V, B)
        threads = os.cpu_count() or 1
        R.lib().ref_set_blas_threads(1)
        t0 = time.perf_counter()
        for _ in range(args.cpu_solves):
            Xc, _ = R.bfs_solve(s, nthreads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": args.cpu_solves / dt, "unit": "solves/s", "cores": threads,
               "kind": "port",
               "sample": f"{args.cpu_solves} full fused FP64 solves of the same system "
                         "(oracle/refcpu.c, OpenBLAS, one OpenMP task per leaf/node)"}
        Xo = Xc[:, : cfg["nrhs"]]
        fwd["mixed_vs_oracle"] = R.rel_error(x_mixed, Xo)
        fwd["fp64_vs_oracle"] = R.rel_error(x_fp64, Xo)
        relres_oracle = {"mixed": R.relres(s, x_mixed), "fp64": R.relres(s, x_fp64),
                         "oracle": R.relres(s, Xo)}

    value = replica_value(ms_mixed, ws)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded Gaussian HODLR system generated on the device, Philox4x32-10)",
        "config": {"workload": f"hodlr_solve N={cfg['N']} leaf={cfg['leaf']} r={cfg['rank']} "
                               f"m={cfg['nrhs']} mixed+refine to relres<=1e-12",
                   **cfg, "levels": int(tree[:, 7].max()), "l2": "inputs 3.5 GB > L2",
                   "parallelism": f"replicas x{ws}"},
        "relres_max": float(max(rrs)), "refine_sweeps": iters,
        "forward_err": fwd, "relres_oracle": relres_oracle,
        "fp64_gpu": {"value": replica_value(ms_fp64, ws), "unit": "solves/s", "ms_per_step": ms_fp64,
                     "relres": rr_fp64,
                     "roofline_frac": solve_frac(ms_fp64, 8, fp64_peak),
                     "tflops": total_flops / (ms_fp64 * 1e-3) / 1e12},
        "mixed_over_fp64": ms_fp64 / ms_mixed,
        "mixed_roofline_frac": solve_frac(ms_mixed, 4, pk["bf16"], passes=3),
        "gflop_per_solve": total_flops / 1e9,
        "roofline": roofline,
        "phases_ms": {"mixed": {k: round(v[0], 4) for k, v in ph_mixed.items()},
                      "fp64": {k: round(v[0], 4) for k, v in ph_fp64.items()}},
        "peaks": {"hbm_gbs": pk["hbm"], "src": pk["src"], "fp64_tflops_nominal": fp64_peak,
                  "fp32_tflops_nominal": fp32_peak},
        "schedules": {"mixed": sched["mixed"], "fp64": sched["fp64"], "autotune": tune_info},
        "gpu_launches": int(launches),
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
