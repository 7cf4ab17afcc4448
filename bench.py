"""Benchmark of the B200 two-site DMRG engine (one JSON line on stdout).

Workload: S=1/2 Heisenberg chain, open boundaries, L=100, J=1, Delta=1, MPO bond
dimension 5, float64; seeded i.i.d. N(0,1) initial MPS with chi=16 (seed 0);
cutoff 1e-12; the chi ramp 32 -> 64 -> 128 -> 256. Synthetic inputs of the
configuration's shapes (no dataset is involved).

  step     = one sweep (left-to-right + right-to-left) at chi = 256, continuing from
             the state left by the W warm-up sweeps (the ramp 32, 64, 128, 256, ...)
  value    = K / (device time of the K timed sweeps)  [sweeps/s], CUDA events on the
             engine's stream, max over ranks
  e2e      = the same K sweeps at chi = 256 through the C ABI from host arrays (the MPO
             and the MPS the warm-up left) to the host energy and final MPS, host wall
             clock, H2D, environment build and D2H included  [sweeps/s]
  roofline = the H_eff contractions (FP64 DMMA): algorithmic flops / their device
             time over the timed sweeps, against a cuBLAS DGEMM measured in the same
             run (no FP64 peak exists in the driver-measured peak file)

  solve    = time to solution through the C ABI: the seeded chi=16 state, the ramp
             32/64/128/256 (three sweeps each), then chi=256 until |dE| < 1e-10

--impl reference runs the oracle (the reference's numpy two-site sweep loop,
restated) on the host cores from the same warm chi=256 state, a few bonds per
step, and reports sweeps/s from the measured per-bond times.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "dmrg-implementations_b200"))

L_SITES = 100
RAMP = [32, 64, 128, 256]
CHI = 256
CUTOFF = 1e-12
KRYLOV = 30
RESTARTS = 2
CPU_BONDS = 14        # bonds of the oracle's sweep in the GPU line's CPU baseline (edge shapes + full width)
BONDS_PER_STEP = 2    # bonds of the oracle's sweep per step of the reference arm
METRIC = "sweeps/s (two-site DMRG, Heisenberg L=100, chi=256, FP64 plain form)"
# DRAM bytes of one H_eff application at chi = 256 (dram__bytes_read.sum + dram__bytes_write.sum
# over its four kernels: step-1 GEMM, MPO mixing, split-K step-3 GEMM, split-K reduce), from one
# ncu capture of `python -m dmrg2.microbench heff --chi 256`; the algorithmic bytes are 9.4 MB
HEFF_TRAFFIC_BYTES_CHI256 = 28.4e6  # ncu DRAM read bytes of the three H_eff kernels at chi=256 (no DRAM writes)


def workload_config(n_gpus, extra=None):
    cfg = {"workload": "heisenberg_xxz_L100_chi256_sweep", "L": L_SITES, "d": 2, "D_mpo": 5,
           "chi": CHI, "warmup_ramp": RAMP, "cutoff": CUTOFF, "krylov_max": KRYLOV,
           "lanczos_restarts": RESTARTS, "init": "N(0,1) chi=16 seed 0 (+rank)",
           "l2": "inputs larger than L2: envs+MPS+Krylov ~0.8 GB resident (L2 126 MB)",
           "parallelism": f"replicas x{n_gpus}"}
    if extra:
        cfg.update(extra)
    return cfg


def schedule(warmup, steps):
    ramp = [RAMP[min(i, len(RAMP) - 1)] for i in range(warmup)]
    return ramp, [CHI] * steps


# ----------------------------------------------------------------------------
# CPU baseline (oracle): the reference's sweep loop, timed bond by bond
# ----------------------------------------------------------------------------
class OracleSweep:
    """The oracle's two-site sweep loop (the reference's numpy primitives restated:
    theta, ARPACK eigsh on H_eff, truncated SVD, environment update), advanced a
    given number of bonds at a time so that a bounded part of a sweep can be timed.

    Starts from an MPS whose sites 1..L-1 are right-canonical (the state a full
    sweep leaves: the GPU run's warm state read back to the host). Building the
    right environments is set-up, not timed. Bonds run in the order of a sweep:
    left to right over bonds 0..L-2, then right to left; both directions cost the
    same per bond shape.
    """

    def __init__(self, mpo, mps, chi, cutoff, krylov_tol=1e-12):
        from oracle import dmrg2_oracle as O
        self.O = O
        self.mpo, self.chi, self.cutoff, self.tol = mpo, chi, cutoff, krylov_tol
        self.A = [a.copy() for a in mps]
        L = self.L = len(mpo)
        dt = np.result_type(self.A[0].dtype, mpo[0].dtype)
        self.Renv = [None] * (L + 1)
        self.Lenv = [None] * (L + 1)
        self.Renv[L] = np.ones((1, 1, 1), dt)
        self.Lenv[0] = np.ones((1, 1, 1), dt)
        for i in range(L - 1, 1, -1):
            self.Renv[i] = O.update_right_env(self.Renv[i + 1], self.A[i], mpo[i])
        self.pos = 0          # bonds done in the current sweep (0 .. 2(L-1))
        self.energy = None
        self.times = {}       # bond shape (chi_left, chi_right), mirrored to sorted order -> seconds

    def bond(self):
        O, A, L = self.O, self.A, self.L
        if self.pos == 2 * (L - 1):
            self.pos = 0
        right = self.pos < L - 1
        i = self.pos if right else 2 * (L - 1) - self.pos - 1
        t0 = time.perf_counter()
        shape = tuple(sorted((A[i].shape[0], A[i + 1].shape[2])))
        theta = np.tensordot(A[i], A[i + 1], axes=(2, 0))
        self.energy, th = O.optimize_two_site(self.Lenv[i], self.Renv[i + 2], self.mpo[i], self.mpo[i + 1],
                                              theta, tol=self.tol)
        cl, d1, d2, cr = th.shape
        U, S, Vh, _ = O.truncated_svd(th.reshape(cl * d1, d2 * cr), self.chi, self.cutoff)
        k = len(S)
        if right:
            A[i] = U.reshape(cl, d1, k)
            A[i + 1] = (S[:, None] * Vh).reshape(k, d2, cr)
            self.Lenv[i + 1] = O.update_left_env(self.Lenv[i], A[i], self.mpo[i])
        else:
            A[i + 1] = Vh.reshape(k, d2, cr)
            A[i] = (U * S).reshape(cl, d1, k)
            self.Renv[i + 1] = O.update_right_env(self.Renv[i + 2], A[i + 1], self.mpo[i + 1])
        self.pos += 1
        self.times.setdefault(shape, []).append(time.perf_counter() - t0)

    def run(self, n_bonds):
        for _ in range(n_bonds):
            self.bond()

    def sweep_seconds(self, dims):
        """Seconds of one full sweep (2 (L-1) bonds) over the bond profile `dims`, from the
        measured time of each bond shape (a shape not run yet counts as the costliest one run)."""
        mean = {k: float(np.mean(v)) for k, v in self.times.items()}
        worst = max(mean.values())
        tot = 0.0
        for i in range(self.L - 1):
            tot += mean.get(tuple(sorted((dims[i], dims[i + 2]))), worst)
        return 2.0 * tot


def oracle_sample(mpo, mps, chi, cutoff, n_bonds):
    """CPU baseline: run the first n_bonds bonds of the oracle's sweep from the given state
    (the left end of the chain up to the full-width middle) and turn the measured per-bond
    times into sweeps/s over the chain's bond-shape profile."""
    t0 = time.perf_counter()
    sw = OracleSweep(mpo, mps, chi, cutoff)
    t1 = time.perf_counter()
    sw.run(n_bonds)
    t2 = time.perf_counter()
    dims = [1] + [a.shape[2] for a in mps]
    return 1.0 / sw.sweep_seconds(dims), {"bonds_run": n_bonds, "timed_s": round(t2 - t1, 2),
                                          "setup_s": round(t1 - t0, 2), "shapes": len(sw.times)}


def cpu_threads():
    return os.cpu_count() or 1


def set_cpu_threads():
    n = str(cpu_threads())
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ.setdefault(k, n)


# ----------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
def measure_dgemm_peak():
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def replica_reduce(values, world, device):
    """Max over ranks of per-rank timings (seconds); the identity on one rank. Every rank
    calls it (the same collective, in the same order)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def replica_throughput(units_per_rank, world, t_max):
    """Whole-job throughput of `world` independent replicas, timed by the slowest one."""
    return world * units_per_rank / t_max


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_ours(args):
    import torch
    import torch.distributed as dist

    import dmrg2
    from dmrg2 import models as P

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    ramp, steady = schedule(args.warmup, args.steps)

    mpo = P.xxz(L_SITES)
    mps = P.random_mps(L_SITES, 2, 16, seed=rank)
    h2d = sum(w.nbytes for w in mpo) + sum(a.nbytes for a in mps)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- warm-up: the chi ramp (untimed); its final MPS is the host state the e2e leg starts from
    eng = dmrg2.DMRG2GPU(L_SITES, 2, CHI, device=local, krylov_max=KRYLOV, max_restarts=RESTARTS,
                         cutoff=CUTOFF, tol=1e-300, min_sweeps=10 ** 6)
    eng.set_mpo(mpo)
    eng.set_mps(mps)
    warm = list(eng.run(schedule=ramp)) if ramp else []
    warm_mps = eng.get_mps()

    # ---- device-timed: K sweeps at chi=256 continuing on the resident state
    launches0 = dmrg2.launch_count()
    barrier()
    torch.cuda.profiler.start()
    with ClockSampler(local) as clocks:
        timed = list(eng.resume(steady))
        barrier()
    torch.cuda.profiler.stop()
    launches = dmrg2.launch_count() - launches0
    energy = eng.get_energy()
    dims = eng.bond_dims()
    eng.close()

    # ---- e2e: the same K sweeps through the C ABI from host arrays (MPO + warm MPS in,
    # energy + final MPS out), host wall clock, H2D/D2H and environment build included
    h2d = sum(w.nbytes for w in mpo) + sum(a.nbytes for a in warm_mps)
    barrier()
    t0 = time.perf_counter()
    eng2 = dmrg2.DMRG2GPU(L_SITES, 2, CHI, device=local, krylov_max=KRYLOV, max_restarts=RESTARTS,
                          cutoff=CUTOFF, tol=1e-300, min_sweeps=10 ** 6)
    t1 = time.perf_counter()
    eng2.set_mpo(mpo)
    eng2.set_mps(warm_mps)
    t2 = time.perf_counter()
    e2e_reports = list(eng2.run(schedule=steady))
    t3 = time.perf_counter()
    final = eng2.get_mps()
    e2e_energy = eng2.get_energy()
    t_e2e = time.perf_counter() - t0
    e2e_phases = {"create": t1 - t0, "set_mpo_mps": t2 - t1, "run": t3 - t2,
                  "env_build": eng2.env_build_seconds(),
                  "sweeps_wall": sum(r["wall_s"] for r in e2e_reports),
                  "sweeps_device": sum(r["device_s"] for r in e2e_reports),
                  "get_mps": t0 + t_e2e - t3}
    eng2.close()
    d2h = sum(a.nbytes for a in final) + 8 * len(e2e_reports)

    dev = sum(r["device_s"] for r in timed)
    heff_s = sum(r["heff_s"] for r in timed)
    heff_fl = sum(r["heff_flops"] for r in timed)
    svd_s = sum(r["svd_s"] for r in timed)
    warm_splits = sum(r["warm_splits"] for r in timed)
    warm_fallbacks = sum(r["warm_fallbacks"] for r in timed)
    eig_fallbacks = sum(r["eig_fallbacks"] for r in timed)
    warm_short = sum(r["warm_short"] for r in timed)
    device_loops = sum(r["device_loops"] for r in timed)
    mv = sum(r["matvecs"] for r in timed)
    n_sw = len(timed)

    # ---- time to solution through the C ABI: the seeded chi=16 state, the 12-sweep ramp
    # 32 -> 64 -> 128 -> 256 (three sweeps each), then chi=256 until |dE| < 1e-10
    barrier()
    solve = c2_solve(mpo, mps, local)
    dev_max, e2e_max, solve_max = replica_reduce([dev, t_e2e, solve["solve_s"]], world, "cuda")
    solve["solve_s"] = solve_max
    peak = measure_dgemm_peak()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    value = replica_throughput(n_sw, world, dev_max)
    achieved = heff_fl / heff_s / 1e12 if heff_s > 0 else 0.0
    set_cpu_threads()
    mv_per_bond = mv / max(1, n_sw * 2 * (L_SITES - 1))
    cpu_value, cpu_info = oracle_sample(mpo, warm_mps, CHI, CUTOFF, n_bonds=CPU_BONDS)
    line = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
        "steps": n_sw, "warmup": len(warm), "ms_per_step": dev_max / n_sw * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded N(0,1) initial MPS, Heisenberg MPO)",
        "config": workload_config(world),
        "energy": energy,
        "max_bond": max(dims),
        "e2e": {"value": replica_throughput(len(e2e_reports), world, e2e_max), "unit": "sweeps/s",
                "h2d_bytes_per_step": h2d // len(e2e_reports), "d2h_bytes_per_step": d2h // len(e2e_reports),
                "energy": e2e_energy,
                # the same sweeps from the same state: the two legs must agree to rounding
                "rel_dE_vs_device_leg": abs(e2e_energy - energy) / max(abs(energy), 1e-300),
                "phases_s": e2e_phases,
                "what": f"{len(e2e_reports)} sweeps at chi={CHI} through dmrg2_create/set_mpo/set_mps/run/get_mps "
                        f"from the host MPS left by the warm-up, host wall clock incl. H2D, environment build, D2H"},
        "roofline": {"kernel": "H_eff contraction (FP64 DMMA GEMMs)", "bound": "tensor",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": HEFF_TRAFFIC_BYTES_CHI256,
                     "traffic_note": "DRAM bytes per H_eff application at chi=256 from an ncu capture of the "
                                     "same kernels; algorithmic bytes 9.4e6 (L, R, theta in and out)",
                     "peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul float64) measured in this run; "
                                    "MEASURED_PEAKS.json has no FP64 figure"},
        "time_share": {"heff": heff_s / dev, "svd": svd_s / dev, "other": max(0.0, 1 - (heff_s + svd_s) / dev)},
        "truncation": {"warm_splits": warm_splits, "warm_short": warm_short, "warm_fallbacks": warm_fallbacks,
                       "eig_fallbacks": eig_fallbacks,
                       "exact_splits": n_sw * 2 * (L_SITES - 1) - warm_splits,
                       "ms_per_bond": 1e3 * svd_s / max(1, n_sw * 2 * (L_SITES - 1))},
        "dominant_kernel": {"name": "truncation (warm-started subspace split: power half-steps, each with unit "
                                    "columns and one triangular CholeskyQR pass; the exact density-matrix split "
                                    "where no warm start applies)",
                            "share": svd_s / dev, "bound": "latency",
                            "ms_per_bond": 1e3 * svd_s / max(1, n_sw * 2 * (L_SITES - 1)),
                            "note": "the inverse Cholesky factor of each k x k Gram matrix is a chain of k "
                                    "dependent pivots in one 8-CTA cluster; no bandwidth or tensor roofline "
                                    "applies"},
        "matvecs_per_bond": mv_per_bond,
        "lanczos_graphs": {"device_loops": device_loops, "solves": n_sw * 2 * (L_SITES - 1),
                           "what": "Lanczos solves of the timed sweeps (restarts counted) that ran as one "
                                   "cached CUDA graph looping over the Krylov steps on the device"},
        "cpu_baseline": {"value": cpu_value, "unit": "sweeps/s", "cores": cpu_threads(), "kind": "port",
                         "sample": f"the oracle's sweep loop (eigsh, SVD, environment update) run over the first "
                                   f"{cpu_info['bonds_run']} bonds of a chi={CHI} sweep from the warm-up's state "
                                   f"({cpu_info['timed_s']} s timed, {cpu_info['shapes']} bond shapes), per-bond "
                                   f"times summed over the chain's bond-shape profile"},
        "solve": solve,
        "clocks": clocks.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    """The reference's CPU path (the oracle port) on this host's cores, same workload and
    metric: the warm chi=256 state of the L=100 chain (the GPU warm-up ramp, run before any
    timing and read back to the host; the oracle's own ramp to chi=256 takes tens of
    minutes), then the oracle's sweep loop, BONDS_PER_STEP bonds per step. W steps warm
    up, K steps are timed; value = sweeps/s from the per-bond times over the chain's
    bond-shape profile (every shape of the chain is run: the left end up to the
    full-width middle, the right end mirrors the left)."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import dmrg2
    from dmrg2 import models as P
    mpo = P.xxz(L_SITES)
    mps = P.random_mps(L_SITES, 2, 16, seed=0)
    ramp, _ = schedule(args.warmup, 0)
    eng = dmrg2.DMRG2GPU(L_SITES, 2, CHI, device=local, krylov_max=KRYLOV, max_restarts=RESTARTS,
                         cutoff=CUTOFF, tol=1e-300, min_sweeps=10 ** 6)
    eng.set_mpo(mpo)
    eng.set_mps(mps)
    eng.run(schedule=ramp)
    warm = eng.get_mps()
    eng.close()
    set_cpu_threads()
    sw = OracleSweep(mpo, warm, CHI, CUTOFF)
    for _ in range(args.warmup):
        sw.run(BONDS_PER_STEP)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sw.run(BONDS_PER_STEP)
    t_timed = time.perf_counter() - t0
    dims = [1] + [a.shape[2] for a in warm]
    value = 1.0 / sw.sweep_seconds(dims)
    n_bonds = (args.warmup + args.steps) * BONDS_PER_STEP
    line = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_timed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(world, {"bonds_per_step": BONDS_PER_STEP}), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": cpu_threads(), "kind": "port",
                         "sample": f"the oracle's sweep loop (the reference's numpy primitives: eigsh, SVD, "
                                   f"environment update) over bonds 0..{n_bonds - 1} of a chi={CHI} sweep of the "
                                   f"L={L_SITES} chain from the warm state, {BONDS_PER_STEP} bonds per step, "
                                   f"{t_timed:.1f} s timed; sweeps/s from the per-bond times over the chain's "
                                   f"bond-shape profile"},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def c2_solve(mpo, mps, device):
    """Seeded chi=16 MPS -> 12-sweep ramp (32, 64, 128, 256; three sweeps each) -> chi=256
    until |dE| < 1e-10, through the C ABI from host arrays: host wall clock with the
    MPO/MPS upload, the environment build and the final MPS read-back included."""
    import dmrg2
    sched = [32] * 3 + [64] * 3 + [128] * 3 + [256] * 3 + [256] * 8
    t0 = time.perf_counter()
    eng = dmrg2.DMRG2GPU(L_SITES, 2, CHI, device=device, krylov_max=KRYLOV, max_restarts=RESTARTS,
                         cutoff=CUTOFF, tol=1e-10, min_sweeps=12)
    eng.set_mpo(mpo)
    eng.set_mps(mps)
    rep = eng.run(schedule=sched)
    final = eng.get_mps()
    e = eng.get_energy()
    wall = time.perf_counter() - t0
    eng.close()
    return {"solve_s": wall, "sweeps": len(rep), "energy": e,
            "last_dE": abs(rep[-1]["energy"] - rep[-2]["energy"]) if len(rep) > 1 else None,
            "device_s": sum(r["device_s"] for r in rep), "final_mps_bytes": int(sum(a.nbytes for a in final)),
            "published_wall_s": {"MI300X dmrg2-gpu (15 sweeps at chi=256, median of 10)": 58.676,
                                 "H100 dmrg2-gpu CUDA port": 23.459},
            "published_energy_chi256": -44.127739893676,
            "what": "L=100 Heisenberg from a seeded chi=16 N(0,1) state: ramp 32/64/128/256 x3 sweeps, then "
                    "chi=256 until |dE| < 1e-10 (stop rule from sweep 12); host wall clock through "
                    "dmrg2_create/set_mpo/set_mps/run/get_mps"}


# ----------------------------------------------------------------------------
# batched and served forms (dmrg2_server_*): solves/s and time-to-converged-energy
# ----------------------------------------------------------------------------
def ramp_to(chi, extra):
    ramp = [c for c in (16, 32, 64, 128, 256) if c < chi] + [chi]
    return ramp + [chi] * extra, len(ramp) + 1


def batched_requests(n=64, seed=7):
    """64 XXZ chains: L in {24,32,48,64}, Delta ~ U[0.5,1.5], J=1, chi_max in {64,128}."""
    from dmrg2 import models as P
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.choice([24, 32, 48, 64]))
        delta = float(rng.uniform(0.5, 1.5))
        chi = int(rng.choice([64, 128]))
        sched, min_sw = ramp_to(chi, 8)
        out.append(dict(mpo=P.xxz(L, delta=delta), mps=P.random_mps(L, 2, 16, seed=int(rng.integers(1 << 30))),
                        schedule=sched, min_sweeps=min_sw, arrival=0.0,
                        desc={"L": L, "delta": round(delta, 4), "chi": chi}))
    return out


def served_requests(n=512, rate=20.0, seed=11):
    """J1-J2 chains (D=8): J1=1, J2 ~ U[0,0.5], L ~ U{16..96}, chi_max in {32,64,128,256};
    Poisson arrivals at `rate` requests/s."""
    from dmrg2 import models as P
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        L = int(rng.integers(16, 97))
        j2 = float(rng.uniform(0.0, 0.5))
        chi = int(rng.choice([32, 64, 128, 256]))
        sched, min_sw = ramp_to(chi, 8)
        out.append(dict(mpo=P.j1j2(L, 1.0, j2), mps=P.random_mps(L, 2, 16, seed=int(rng.integers(1 << 30))),
                        schedule=sched, min_sweeps=min_sw, arrival=t,
                        desc={"L": L, "J2": round(j2, 4), "chi": chi}))
    return out


def serve(reqs, max_active, device, timed_arrivals):
    """Submit reqs to a server (at their arrival times when timed_arrivals), wait for all."""
    import dmrg2
    srv = dmrg2.Server(device=device, max_active=max_active)
    t0 = time.perf_counter()
    ids = []
    for r in reqs:
        if timed_arrivals:
            dt = r["arrival"] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
        ids.append(srv.submit(r["mpo"], r["schedule"], mps=r["mps"], tol=1e-10, min_sweeps=r["min_sweeps"],
                              krylov_max=KRYLOV, max_restarts=RESTARTS, cutoff=1e-12))
    res = [srv.result(i) for i in ids]
    wall = time.perf_counter() - t0
    srv.close()
    return res, wall


def run_server_workload(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if args.workload == "batched":
        reqs = batched_requests(args.requests or 64)
        timed = False
        metric = "solves/s (64 XXZ chains, L in {24..64}, chi_max in {64,128}, FP64, continuous admission)"
    else:
        reqs = served_requests(args.requests or 512, rate=args.rate)
        timed = True
        metric = ("solves/s (J1-J2 D=8 request stream, Poisson %g req/s, L in 16..96, chi_max in {32..256}, FP64)"
                  % args.rate)
    n_plain = min(len(reqs), args.plain_sample)
    # the plain form: the same requests one at a time, back to back (no arrival gaps)
    plain, plain_wall = serve(reqs[:n_plain], 1, local, False)
    with ClockSampler(local) as clocks:
        res, wall = serve(reqs, args.max_active, local, timed)
    import dmrg2
    failed = [r["message"] for r in res if r["state"] != dmrg2.REQ_DONE]
    lat = np.array([r["t_done"] - r["t_submit"] for r in res])
    span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    dE = max(abs(a["energy"] - b["energy"]) / abs(b["energy"]) for a, b in zip(res[:n_plain], plain))
    plain_rate = n_plain / sum(r["t_done"] - r["t_admit"] for r in plain)
    value = len(res) / span
    line = {
        "metric": metric, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": len(res), "warmup": 0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded MPOs and N(0,1) initial MPS)", "impl": "ours",
        "config": {"workload": args.workload, "requests": len(res), "max_active": args.max_active,
                   "arrival_rate_per_s": args.rate if args.workload == "served" else None,
                   "schedule": "ramp 16,32,.. to chi_max then chi_max x8, stop |dE| < 1e-10",
                   "krylov_max": KRYLOV, "cutoff": 1e-12},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "plain": {"solves_per_s": plain_rate, "requests": n_plain,
                  "what": "the same requests solved one at a time on one stream (sum of solve times)"},
        "speedup_vs_plain": value / plain_rate,
        "max_rel_dE_mix_vs_alone": dE, "failed": len(failed),
        "mean_sweeps": float(np.mean([r["sweeps"] for r in res])),
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line))


# ----------------------------------------------------------------------------
# precision form: Josephson array, plain FP64 vs split-BF16 matvecs
# ----------------------------------------------------------------------------
def run_precision_workload(args):
    """Josephson junction array L=24, d=5 (n in -2..2), E_C=1, E_J=2, n_g=0.25,
    A=2 pi 0.1/L, D=4, complex128; seeded complex Gaussian chi=16 start, chi_max=128,
    10 sweeps; the plain form, the precision form and the plain form with the randomised
    split (truncation mode 2) on the same inputs."""
    import torch
    import dmrg2
    from dmrg2 import models as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    L, nmax, chi = 24, 2, 128
    mpo = P.josephson(L, n_max=nmax, E_J=2.0, E_C=1.0, n_g=0.25, phi=2 * np.pi * 0.1 / L, onsite="shifted")
    mps = P.random_mps(L, 2 * nmax + 1, 16, seed=0, dtype=np.complex128)
    nop = np.diag(np.arange(2 * nmax + 1) - float(nmax)).astype(np.complex128)
    sched = [chi] * (args.steps if args.steps != 3 else 10)
    out = {}
    for name, prec, trunc in (("plain", 0, 0), ("split", 1, 0), ("rsvd", 0, 2)):
        eng = dmrg2.DMRG2GPU(L, 2 * nmax + 1, chi, dtype=np.complex128, krylov_max=KRYLOV, max_restarts=RESTARTS,
                             cutoff=1e-12, tol=1e-300, min_sweeps=10 ** 6, precision=prec, truncation=trunc,
                             device=local)
        eng.set_mpo(mpo)
        eng.set_mps(mps)
        rep = eng.run(schedule=sched)
        out[name] = {"energy": rep[-1]["energy"], "device_s": sum(r["device_s"] for r in rep),
                     "heff_s": sum(r["heff_s"] for r in rep), "svd_s": sum(r["svd_s"] for r in rep),
                     "matvecs": sum(r["matvecs"] for r in rep),
                     "lowprec_matvecs": sum(r["lowprec_matvecs"] for r in rep),
                     "rsvd_splits": sum(r["rsvd_splits"] for r in rep),
                     "trunc_err_max": rep[-1]["trunc_err_max"],
                     "n": eng.expect_local(nop), "max_bond": max(eng.bond_dims())}
        eng.close()
    p, q, z = out["plain"], out["split"], out["rsvd"]
    bonds = len(sched) * 2 * (L - 1)
    line = {
        "metric": "sweeps/s (Josephson L=24 d=5 chi=128 complex128, precision form vs FP64 plain form)",
        "value": len(sched) / q["device_s"], "unit": "sweeps/s", "n_gpus": 1, "steps": len(sched), "warmup": 0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (split-bf16 matvecs)",
        "data": "synthetic (seeded complex Gaussian MPS, Josephson MPO)", "impl": "ours",
        "config": {"workload": "josephson_L24_d5_chi128_precision", "E_C": 1.0, "E_J": 2.0, "n_g": 0.25,
                   "A": "2 pi 0.1 / L", "sweeps": len(sched), "cutoff": 1e-12, "krylov_max": KRYLOV},
        "plain": {"sweeps_per_s": len(sched) / p["device_s"], "energy": p["energy"], "matvecs": p["matvecs"],
                  "heff_s": p["heff_s"], "svd_s": p["svd_s"]},
        "split": {"sweeps_per_s": len(sched) / q["device_s"], "energy": q["energy"], "matvecs": q["matvecs"],
                  "lowprec_matvecs": q["lowprec_matvecs"], "heff_s": q["heff_s"], "svd_s": q["svd_s"]},
        "rsvd": {"sweeps_per_s": len(sched) / z["device_s"], "energy": z["energy"], "svd_s": z["svd_s"],
                 "truncation_ms_per_bond": 1e3 * z["svd_s"] / bonds, "rsvd_splits": z["rsvd_splits"],
                 "trunc_err_max": z["trunc_err_max"],
                 "rel_dE_vs_fp64": abs(z["energy"] - p["energy"]) / abs(p["energy"]),
                 "what": "plain form with the randomised split (r = k + 10 sketch, shifted CholeskyQR3) "
                         "where it applies; the plain form's truncation is the default one: the exact "
                         "density-matrix split on the first sweep at a cap, the warm-started split "
                         "(complex CholeskyQR on the real embedding) on sweeps that repeat it"},
        "plain_truncation_ms_per_bond": 1e3 * p["svd_s"] / bonds, "plain_trunc_err_max": p["trunc_err_max"],
        "rel_dE_split_vs_fp64": abs(q["energy"] - p["energy"]) / abs(p["energy"]),
        "max_abs_dn_split_vs_fp64": float(np.max(np.abs(np.asarray(q["n"]) - np.asarray(p["n"])))),
        "max_bond": q["max_bond"],
    }
    if rank == 0:
        print(json.dumps(line))


def run_pdmrg_workload(args):
    """Parallel segmented sweeps (dmrg2_pdmrg_run) on the sweep workload's state: Heisenberg
    L=100, chi=256, from the state a 12-sweep ramp 32/64/128/256 (x3) leaves. Plain
    sweeps continue from that state, and the parallel driver runs P = 2, 4, 8 segments
    (one full warm-up sweep, n_local = 1); an outer iteration sweeps every segment both ways
    and merges every boundary once, i.e. one sweep's worth of bonds. Reports
    sweep-equivalents/s over the outer iterations after the first."""
    import torch
    import dmrg2
    from dmrg2 import models as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    mpo = P.xxz(L_SITES, delta=1.0)
    kw = dict(device=local, krylov_max=KRYLOV, max_restarts=RESTARTS, cutoff=CUTOFF, tol=1e-300,
              min_sweeps=10 ** 6)
    eng = dmrg2.DMRG2GPU(L_SITES, 2, CHI, **kw)
    eng.set_mpo(mpo)
    eng.set_mps(P.random_mps(L_SITES, 2, 16, seed=0))
    eng.run(schedule=[c for c in RAMP for _ in range(3)])
    state = eng.get_mps()
    plain = eng.resume([CHI] * 4)
    t_plain = float(np.median([r["device_s"] for r in plain[1:]]))
    e_plain = plain[-1]["energy"]
    eng.close()
    rows = {}
    for nseg in (2, 4, 8):
        e2 = dmrg2.DMRG2GPU(L_SITES, 2, CHI, **kw)
        e2.set_mpo(mpo)
        e2.set_mps(state)
        rep = e2.pdmrg(n_segments=nseg, n_outer=4, n_local=1, n_warmup=1)
        outer = [r for r in rep if r["phase"] == 2]
        t = float(np.median([r["wall_s"] for r in outer[1:]])) if len(outer) > 1 else outer[0]["wall_s"]
        rows[nseg] = {"s_per_outer": t, "sweep_equivalents_per_s": 1.0 / t, "outer_iterations": len(outer),
                      "energy": e2.get_energy(), "rel_dE_vs_plain": abs(e2.get_energy() - e_plain) / abs(e_plain),
                      "matvecs": sum(r["matvecs"] for r in outer), "svd_s": sum(r["svd_s"] for r in outer)}
        e2.close()
    best = max(rows, key=lambda k: rows[k]["sweep_equivalents_per_s"])
    line = {
        "metric": "sweep-equivalents/s (parallel segmented sweeps, Heisenberg L=100, chi=256, FP64)",
        "value": rows[best]["sweep_equivalents_per_s"], "unit": "sweeps/s", "n_gpus": 1, "steps": 4, "warmup": 12,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded N(0,1) initial MPS, Heisenberg MPO)", "impl": "ours",
        "config": {"workload": "pdmrg_heisenberg_L100_chi256", "segments": sorted(rows), "n_local": 1,
                   "start": "state after the ramp 32/64/128/256 x3, one full warm-up sweep", "best_segments": best},
        "plain": {"sweeps_per_s": 1.0 / t_plain, "energy": e_plain, "what": "four more plain sweeps, device time"},
        "segments": rows,
    }
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["sweep", "batched", "served", "precision", "pdmrg"], default="sweep")
    ap.add_argument("--requests", type=int, default=0)
    ap.add_argument("--rate", type=float, default=20.0, help="served workload: Poisson arrivals per second")
    ap.add_argument("--max-active", type=int, default=12)
    ap.add_argument("--plain-sample", type=int, default=24)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "precision" and args.impl == "ours":
        run_precision_workload(args)
    elif args.workload == "pdmrg" and args.impl == "ours":
        run_pdmrg_workload(args)
    elif args.workload != "sweep" and args.impl == "ours":
        run_server_workload(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
