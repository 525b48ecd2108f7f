#!/usr/bin/env python
"""Benchmark: batched VMC electron moves per second on one B200 (per GPU, weak scaling).

Workload (default): the C2-like pseudopotential dimer (8 electrons, 60 contracted
Gaussians, one determinant, e-e/e-n/e-e-n Jastrow, 12-point nonlocal quadrature) with
8192 walkers in one launch, mixed precision.  A step is one VMC sweep over all walkers:
8 single-electron Metropolis proposals per walker (ratio, accept, Sherman-Morrison and
Jastrow-table update) plus one full local-energy evaluation per walker, including the
nonlocal pseudopotential quadrature.  e-moves/s = walkers x electrons x steps / time.

Output: one JSON line (rank 0).  --impl reference times the CPU restatement of the
reference algorithm (the reference itself is Fortran and cannot be built here) on the
host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "e-moves/s & param-grad samples/s: mixed vs FP64, 1 B200, |ΔE_L|≤1e-6 Ha"
UNIT = "e-moves/s"
SEED = 20261203


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--system", type=int, default=2)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--walkers", type=int, default=0)
    ap.add_argument("--step-size", type=float, default=0.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-arm", action="store_true")
    ap.add_argument("--no-cluster", action="store_true", help="skip the 128-electron cluster measurement")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [q.strip() for q in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes per walker of one k_vmc launch, from a full ncu capture of one launch
# (2048 walkers, mixed precision: 6.88 MB read + 0.17 MB
# written); the traffic grows with the walker count, so a full launch is scaled by walkers.
KVMC_DRAM_BYTES_PER_WALKER = {(2, "mixed"): (6.883072e6 + 0.165888e6) / 2048}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def state_bytes(system, precision):
    """Algorithmic HBM bytes per walker per sweep: the persistent walker state (positions,
    reference-determinant inverses, Jastrow pair table, ln|D|, sign, J) read and written once."""
    N, nup = system.nelec, system.nup
    ndn = N - nup
    t = 8 if precision == "fp64" else 4
    b = 8 * 3 * N + 8 * (nup * nup + ndn * ndn) + t * N * N + 8 * 3
    return 2 * b


def cpu_baseline_sample(system, seconds=12.0):
    """Oracle (CPU restatement, OpenMP over walkers, all host threads) on a bounded sample."""
    from oracle.oracle import Oracle
    o = Oracle(system)
    ncores = os.cpu_count() or 1
    nw = max(ncores * 4, 32)
    x = system_walkers(system, nw, seed=3)
    t0 = time.perf_counter()
    o.vmc(x, 1, seed=SEED, sweep0=0, step=step_size(system), nthreads=ncores)
    dt1 = max(time.perf_counter() - t0, 1e-3)
    nsw = max(1, int(seconds / dt1))
    t0 = time.perf_counter()
    o.vmc(x, nsw, seed=SEED, sweep0=1, step=step_size(system), nthreads=ncores)
    dt = time.perf_counter() - t0
    v = nw * system.nelec * nsw / dt
    return {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
            "sample": f"{nw} walkers x {nsw} sweeps of {system.name} on the FP64 oracle ({dt:.1f} s)"}


def system_walkers(system, nw, seed):
    from champ_b200.system import initial_walkers
    return initial_walkers(system, nw, seed=seed)


def step_size(system):
    return ARGS.step_size if ARGS.step_size > 0 else system.step


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference(args, system, rank, world):
    if rank != 0:
        return
    from oracle.oracle import Oracle
    o = Oracle(system)
    ncores = os.cpu_count() or 1
    nw = max(ncores * 4, 32)
    x = system_walkers(system, nw, seed=3)
    for i in range(args.warmup):
        r = o.vmc(x, 1, seed=SEED, sweep0=i, step=step_size(system), nthreads=ncores)
        x = r["x"]
    t0 = time.perf_counter()
    for k in range(args.steps):
        r = o.vmc(x, 1, seed=SEED, sweep0=args.warmup + k, step=step_size(system), nthreads=ncores)
        x = r["x"]
    dt = time.perf_counter() - t0
    v = nw * system.nelec * args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config_of(system, nw, "fp64"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                             "sample": f"{nw} walkers per step, 1 sweep each, FP64 CPU restatement of the reference "
                                       f"algorithm (the Fortran reference cannot be compiled here)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_of(system, nw, prec):
    return {"workload": f"{system.name}: VMC sweeps, {system.nelec} electrons, {system.nbasis} basis functions, "
                        f"{system.ndet} determinant(s), {system.ncent} centres, "
                        f"{'12-point NLPP quadrature' if system.nloc else 'all-electron'}",
            "walkers_per_gpu": nw, "electrons": system.nelec, "precision": prec,
            "step": "one sweep: N single-electron proposals per walker + full E_L",
            "l2": "flushed between timed steps (256 MB write)"}


def lib_accumulate(eng):
    """champ_accumulate_oh with the results left on the device (no host copies)."""
    import ctypes as C
    return eng.lib.champ_accumulate_oh(eng.h, None, None, None)


def time_engine(eng, system, args, nsteps, nwarm, flush, torch, sweep_base):
    st = step_size(system)
    for i in range(nwarm):
        eng.vmc_sweeps(1, SEED, sweep0=sweep_base + i, step=st, stats=False)
    torch.cuda.synchronize()
    evs = []
    for k in range(nsteps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.vmc_sweeps(1, SEED, sweep0=sweep_base + nwarm + k, step=st, stats=False)
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)  # ms


def allmax(x, world, torch, dist):
    """Max over ranks of a per-rank number (every rank calls this in the same order)."""
    from champ_b200.dist import max_over_ranks
    return max_over_ranks(x)


def time_param_grad(eng, system, nsteps, flush, torch):
    """d ln psi/dp and dE_L/dp for every walker, folded into the FP64 O/H accumulators (one
    champ_param_grad + champ_accumulate_oh per step, and with several ranks the all-reduce of
    the accumulators, the one exchange step of the path); the walkers move by one VMC sweep
    between steps, outside the timed events.  Returns ms for nsteps."""
    from champ_b200.dist import reduce_oh, rank_world
    multi = rank_world()[1] > 1
    tpg = 0.0
    for k in range(nsteps + 2):
        eng.vmc_sweeps(1, SEED, sweep0=30000 + k, step=step_size(system), stats=False)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.param_grad(host=False)
        eng._check(lib_accumulate(eng))
        if multi:
            reduce_oh(eng)
        e1.record()
        torch.cuda.synchronize()
        if k >= 2:
            tpg += e0.elapsed_time(e1)
    return tpg


def measure(system, nw, prec, steps, warmup, pg_steps, rank, world, flush, torch, dist, fp64_arm=True):
    """e-moves/s of the fused VMC sweep (mixed or FP64), the FP64 arm of the same workload,
    param-grad samples/s in both precisions and the mixed-precision E_L error on the same walkers."""
    from champ_b200.engine import Engine
    eng = Engine(system, nw, prec)
    eng.set_walkers(system_walkers(system, nw, seed=1000 + rank))
    eng.vmc_sweeps(10, SEED + rank, sweep0=0, step=step_size(system), stats=False)  # equilibration
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clk.start()
    time.sleep(0.5)  # let the sampler start before the timed region
    t_wall = time.perf_counter()
    ms = time_engine(eng, system, None, steps, warmup, flush, torch, 100)
    t_wall = time.perf_counter() - t_wall
    clocks = clk.stop()
    ms = allmax(ms, world, torch, dist)
    out = {"value": nw * world * system.nelec * steps / (ms * 1e-3), "ms_per_step": ms / steps,
           "clocks": clocks, "wall_s_timed_region": t_wall,
           "launches_per_step": eng.get_option("launches_per_sweep")}
    nj, ncsf, norb = eng.nparam()
    npar = {"jastrow": nj, "csf": ncsf, "orbital": norb}
    tpg = allmax(time_param_grad(eng, system, pg_steps, flush, torch), world, torch, dist)
    out["param_grad"] = {"value": nw * world * pg_steps / (tpg * 1e-3), "unit": "param-grad samples/s",
                         "n_params": nj + ncsf + norb, "params": npar, "ms_per_step": tpg / pg_steps,
                         "step": "d ln psi/dp and dE_L/dp for all walkers + FP64 O/H accumulation (cuBLAS DGEMM)"}
    if prec == "mixed" and fp64_arm:
        eng64 = Engine(system, nw, "fp64")
        xw = eng.get_walkers()
        eng64.set_walkers(xw)
        n64 = max(3, steps // 4)
        ms64 = allmax(time_engine(eng64, system, None, n64, 2, flush, torch, 10000), world, torch, dist)
        v64 = nw * world * system.nelec * n64 / (ms64 * 1e-3)
        pg64 = max(2, pg_steps // 2)
        tpg64 = allmax(time_param_grad(eng64, system, pg64, flush, torch), world, torch, dist)
        vpg64 = nw * world * pg64 / (tpg64 * 1e-3)
        # mixed-precision error of E_L on identical walkers (same quadrature rotation)
        eng.set_walkers(xw)
        eng64.set_walkers(xw)
        em, e64 = eng.eval_full(), eng64.eval_full()
        sd = em["energy"] - e64["energy"]
        d = np.abs(sd)
        sc = np.maximum(1.0, np.maximum(np.abs(e64["energy"]), np.abs(e64["d2lnpsi"])))
        out["fp64_arm"] = {"value": v64, "unit": UNIT, "ms_per_step": ms64 / n64, "mixed_over_fp64": out["value"] / v64,
                           "param_grad": {"value": vpg64, "unit": "param-grad samples/s", "ms_per_step": tpg64 / pg64,
                                          "mixed_over_fp64": out["param_grad"]["value"] / vpg64}}
        out["mixed_error"] = {"max_abs_dEL_Ha": float(d.max()), "median_abs_dEL_Ha": float(np.median(d)),
                              "frac_samples_within_1e-6_Ha": float(np.mean(d <= 1e-6)),
                              "max_rel_to_max(1,|E_L|,|lap ln psi|)": float(np.max(d / sc)),
                              "mean_dEL_Ha": float(sd.mean()), "mean_dEL_stderr_Ha": float(sd.std() / np.sqrt(len(sd))),
                              "walkers": nw}
        eng64.close()
    out["_eng"] = eng
    return out


def measure_dmc(system, target, nstep, torch):
    """DMC throughput of the DMC workload: drift-diffusion moves (two gradient evaluations per
    proposal), E_L, reweighting and branching for the whole population per step, steps replayed
    as CUDA graphs; e-moves/s = sum over steps of population x electrons / device time."""
    from champ_b200.engine import Engine
    eng = Engine(system, int(1.6 * target), "mixed")
    eng.set_walkers(system_walkers(system, target, seed=11))
    eng.vmc_sweeps(20, SEED, sweep0=0, step=step_size(system), stats=False)
    eng.dmc_init(target, 0.01)
    eng.dmc_steps(20, seed=SEED)  # equilibration, graph capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    st = eng.dmc_steps(nstep, seed=SEED)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    moves = float(st[:, 0].sum()) * system.nelec
    eng.close()
    return {"workload": f"{system.name}: DMC, target population {target}, tau 0.01", "value": moves / (ms * 1e-3),
            "unit": UNIT, "ms_per_step": ms / nstep, "steps": nstep,
            "population": [float(st[:, 0].min()), float(st[:, 0].max())],
            "step": "per walker: N drift-diffusion proposals (gradient before and after), Green's-function "
                    "acceptance, updates; E_L with NLPP; reweighting; branching; one CUDA graph per two steps",
            "note": "the timed call includes one device-to-host copy of the step statistics and population"}


def mixed_error_of(system, nw, seed=5):
    """|E_L(mixed) - E_L(FP64)| on identical walkers of one system (eval_full of both engines)."""
    from champ_b200.engine import Engine
    x = system_walkers(system, nw, seed=seed)
    em, e64 = Engine(system, nw, "mixed"), Engine(system, nw, "fp64")
    em.set_walkers(x)
    e64.set_walkers(x)
    em.vmc_sweeps(20, SEED, sweep0=0, step=step_size(system), stats=False)  # equilibrate the mixed walkers
    xw = em.get_walkers()
    em.set_walkers(xw)
    e64.set_walkers(xw)
    a, b = em.eval_full(), e64.eval_full()
    sd = a["energy"] - b["energy"]
    d = np.abs(sd)
    # per sample, and on the estimator: the walker average of E_L(mixed) - E_L(FP64) (its bias)
    out = {"system": system.name, "walkers": nw, "max_abs_dEL_Ha": float(d.max()), "median_abs_dEL_Ha": float(np.median(d)),
           "frac_samples_within_1e-6_Ha": float(np.mean(d <= 1e-6)), "mean_dEL_Ha": float(sd.mean()),
           "mean_dEL_stderr_Ha": float(sd.std() / np.sqrt(len(sd)))}
    em.close()
    e64.close()
    return out


def main():
    global ARGS
    args = ARGS = parse()
    from champ_b200 import system as S
    system = S.get_system(args.system)
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, system, rank, world)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    nw = args.walkers or system.walkers
    prec = args.precision
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    m = measure(system, nw, prec, args.steps, args.warmup, max(3, args.steps // 20), rank, world, flush, torch, dist,
                fp64_arm=not args.no_fp64_arm)
    eng = m.pop("_eng")
    value, ms_step = m["value"], m["ms_per_step"]
    # roofline of the dominant kernel (the fused sweep kernel, one launch per step)
    peaks, peak_kind = measured_peaks()
    alg_bytes = state_bytes(system, prec) * nw
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    tpw = KVMC_DRAM_BYTES_PER_WALKER.get((args.system, prec))
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": (tpw * nw) if tpw else None,
            "traffic_source": "ncu dram__bytes_read+write of one 2048-walker launch, per walker x walkers"
            if tpw else None, "algorithmic_bytes": alg_bytes, "peak_source": peak_kind,
            "kernel": "k_vmc (fused sweep)",
            "note": "algorithmic bytes = persistent walker state read+written once per sweep; the kernel is "
                    "CUDA-core bound (see profiles/), so this fraction is small by construction"}
    # end to end through the host-facing call: walkers in from pinned host memory, one sweep,
    # E_L and walkers back to host memory, every step
    xh = torch.empty((nw, system.nelec, 3), dtype=torch.float64, pin_memory=True)
    xh.copy_(torch.from_numpy(eng.get_walkers()))
    elh = torch.empty((nw,), dtype=torch.float64, pin_memory=True)
    import ctypes as C
    from champ_b200.engine import load_library
    lib = load_library()
    px = C.cast(xh.data_ptr(), C.POINTER(C.c_double))
    pel = C.cast(elh.data_ptr(), C.POINTER(C.c_double))
    for i in range(2):
        eng._check(lib.champ_vmc_run_host(eng.h, nw, px, 1, SEED, 20000 + i, step_size(system), pel))
    if world > 1:
        dist.barrier()
    ne2e = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for k in range(ne2e):
        eng._check(lib.champ_vmc_run_host(eng.h, nw, px, 1, SEED, 20010 + k, step_size(system), pel))
    te2e = allmax(time.perf_counter() - t0, world, torch, dist)
    e2e = {"value": nw * world * system.nelec * ne2e / te2e, "unit": UNIT,
           "h2d_bytes_per_step": nw * system.nelec * 3 * 8, "d2h_bytes_per_step": nw * system.nelec * 3 * 8 + nw * 8,
           "call": "champ_vmc_run_host (walkers host->device, state rebuild, 1 sweep, E_L and walkers device->host)"}
    eng.close()
    # the 128-electron cluster, where the mixed-vs-FP64 target is set (4096 walkers)
    big = None
    if args.system != 5 and not args.no_cluster:
        s5 = S.get_system(5)
        b = measure(s5, s5.walkers, "mixed", max(6, args.steps // 100), 2, 2, rank, world, flush, torch, dist)
        b.pop("_eng").close()
        big = {"workload": config_of(s5, s5.walkers, "mixed")["workload"], "walkers_per_gpu": s5.walkers, **b}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            big["cpu_baseline"] = cpu_baseline_sample(s5, seconds=8.0)
    dmc = None
    if args.system != 4 and not args.no_cluster and world == 1:
        s4 = S.get_system(4)
        dmc = measure_dmc(s4, s4.walkers, max(10, args.steps // 20), torch)
    # the same error on a physical wave function (the reference's Be example: 4 determinants,
    # Slater basis, optimised Jastrow), where E_L varies little between samples
    phys = mixed_error_of(S.be_example(), 4096) if prec == "mixed" else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(system)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
                "config": config_of(system, nw, prec), "clocks": m["clocks"],
                "gpu_launches": args.steps * m["launches_per_step"],
                "roofline": roof, "fp64_arm": m.get("fp64_arm"), "param_grad": m["param_grad"],
                "mixed_error": m.get("mixed_error"), "mixed_error_physical": phys, "e2e": e2e, "cpu_baseline": cpu,
                "wall_s_timed_region": m["wall_s_timed_region"], "cluster128": big, "dmc": dmc}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
