#!/usr/bin/env python
"""Benchmark: batched VMC electron moves per second and parameter-gradient samples per second,
mixed precision against FP64, on one B200 (per GPU, weak scaling).

Headline workload (system 5): 32 pseudo-atoms (Z_eff 4) in a 14-bohr cube, 64 + 64 electrons,
416 contracted Gaussians, one determinant, e-e/e-n/e-e-n Jastrow, 12-point nonlocal quadrature,
4096 walkers in one launch.  A step is one VMC sweep over all walkers: 128 single-electron
Metropolis proposals per walker (ratio, accept, Sherman-Morrison and Jastrow-table update) plus one
full local-energy evaluation per walker including the nonlocal quadrature.
e-moves/s = walkers x electrons x steps / device time.  Mixed precision runs the moves in FP32
and every full evaluation in FP64, so each sample's E_L equals the FP64 engine's (|dE_L| <= 1e-6 Ha,
measured here on identical walkers).  Beside it: the FP64 engine, the FP32 engine (FP32 full
evaluation, tensor-core orbitals; it does not meet the 1e-6 Ha bound, its error is reported),
parameter-gradient samples/s, the other benchmark systems, and the CPU restatement of the
reference algorithm on the host cores.

Output: one JSON line (rank 0).  --impl reference times the CPU restatement of the reference
algorithm (the reference itself is Fortran and cannot be built here) on the host cores.
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
NSM = 148                       # B200 streaming multiprocessors
FMA_PER_SM_CLK = {"fp64": 64, "fp32": 128}  # FP64 / FP32 fused multiply-adds per SM per clock

# Executed floating-point operations per walker of one sweep phase (2 per FMA, 1 per add/mul, 512
# per DMMA m8n8k4 warp instruction), counted by ncu (smsp__sass_thread_inst_executed_op_{d,f}{fma,
# add,mul}_pred_on.sum, sm__inst_executed_pipe_tensor_subpipe_dmma.sum) on a 256-walker sweep of
# the same kernels and divided by the walkers (profiles/flops_cluster128.md).  "eval" is the FP64
# full evaluation (k_el_jas, k_el_orb, k_el_inv, k_el_fin); None until counted: the roofline's
# achieved figure is then left out.
FLOPS_PER_WALKER = {
    ("cluster128", "eval", "fp64"): 250.86e6,     # CUDA cores 216.31 M + DMMA 34.55 M
    ("cluster128", "moves", "fp32"): 18.54e6,     # FP32 (plus 2.85 M FP64: the Sherman-Morrison updates)
    ("cluster128", "sweep", "fp64"): None,
}
# DRAM bytes per walker of the same launches (dram__bytes_read.sum + dram__bytes_write.sum).
DRAM_PER_WALKER = {
    ("cluster128", "eval", "fp64"): 1555342.0,    # 218.0 MB read + 180.3 MB written / 256
    ("cluster128", "moves", "fp32"): 162209.0,    # 39.8 MB read + 1.8 MB written / 256
    ("cluster128", "sweep", "fp64"): None,
}

def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--system", type=int, default=5)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "fp32"])
    ap.add_argument("--walkers", type=int, default=0)
    ap.add_argument("--step-size", type=float, default=0.0)
    ap.add_argument("--quick", action="store_true", help="headline only: no other systems, arms or baselines")
    ap.add_argument("--no-cpu-baseline", action="store_true")
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


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def system_walkers(system, nw, seed):
    from champ_b200.system import initial_walkers
    return initial_walkers(system, nw, seed=seed)


def step_size(system):
    return ARGS.step_size if ARGS.step_size > 0 else system.step


def dist_setup():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def allmax(x):
    from champ_b200.dist import max_over_ranks
    return max_over_ranks(x)


def config_of(system, nw, prec):
    return {"workload": f"{system.name}: VMC sweeps, {system.nelec} electrons, {system.nbasis} basis functions, "
                        f"{system.ndet} determinant(s), {system.ncent} centres, "
                        f"{f'{system.nquad}-point NLPP quadrature' if system.nloc else 'all-electron'}",
            "walkers_per_gpu": nw, "electrons": system.nelec, "precision": prec,
            "step": "one sweep: N single-electron proposals per walker + full E_L",
            "l2": "flushed between timed steps (256 MB write)"}


# ---------------------------------------------------------------------------------------------
# CPU: the oracle (FP64 restatement of the reference algorithm), OpenMP over walkers
# ---------------------------------------------------------------------------------------------
def cpu_sample(system, seconds):
    """Oracle VMC on a bounded sample of the workload, all host threads: multi-sweep calls."""
    from oracle.oracle import Oracle
    o = Oracle(system)
    ncores = os.cpu_count() or 1
    nw = max(ncores * 4, 32)
    x = system_walkers(system, nw, seed=3)
    t0 = time.perf_counter()
    r = o.vmc(x, 1, seed=SEED, sweep0=0, step=step_size(system), nthreads=ncores)
    dt1 = max(time.perf_counter() - t0, 1e-3)
    nsw = max(1, int(seconds / dt1))
    t0 = time.perf_counter()
    o.vmc(r["x"], nsw, seed=SEED, sweep0=1, step=step_size(system), nthreads=ncores)
    dt = time.perf_counter() - t0
    return {"value": nw * system.nelec * nsw / dt, "unit": UNIT, "cores": ncores, "kind": "port",
            "sample": f"{nw} walkers x {nsw} sweeps of {system.name} in one call on the FP64 oracle ({dt:.1f} s)"}


def run_reference(args, system, rank, world):
    """The reference algorithm's CPU path (the oracle), all host threads, on the headline config:
    each step one call of several sweeps on a bounded walker sample."""
    if rank != 0:
        return
    from oracle.oracle import Oracle
    o = Oracle(system)
    ncores = os.cpu_count() or 1
    nw = max(ncores * 4, 32)
    x = system_walkers(system, nw, seed=3)
    t0 = time.perf_counter()
    r = o.vmc(x, 1, seed=SEED, sweep0=0, step=step_size(system), nthreads=ncores)
    per_sweep = max(time.perf_counter() - t0, 1e-4)
    nsw = max(1, min(50, int(4.0 / per_sweep)))  # a step of about 4 s or at most 50 sweeps
    x = r["x"]
    for i in range(args.warmup):
        x = o.vmc(x, 1, seed=SEED, sweep0=1 + i, step=step_size(system), nthreads=ncores)["x"]
    t0 = time.perf_counter()
    for k in range(args.steps):
        x = o.vmc(x, nsw, seed=SEED, sweep0=100 + k * nsw, step=step_size(system), nthreads=ncores)["x"]
    dt = time.perf_counter() - t0
    v = nw * system.nelec * nsw * args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference", "config": config_of(system, nw, "fp64"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                             "sample": f"per step: {nw} walkers x {nsw} sweeps in one call, FP64 CPU restatement of "
                                       f"the reference algorithm (the Fortran reference cannot be compiled here)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# GPU measurements
# ---------------------------------------------------------------------------------------------
def time_sweeps(eng, system, nsteps, nwarm, flush, torch, sweep_base):
    """Device ms of nsteps VMC sweeps (one champ_vmc_sweeps call each, L2 flushed before each),
    and the per-phase kernel times inside them."""
    st = step_size(system)
    for i in range(nwarm):
        eng.vmc_sweeps(1, SEED, sweep0=sweep_base + i, step=st, stats=False)
    torch.cuda.synchronize()
    eng.set_option("phase_timing", 1)
    eng.phase_times()
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
    ph = eng.phase_times()
    eng.set_option("phase_timing", 0)
    return sum(a.elapsed_time(b) for a, b in evs), ph


def time_param_grad(eng, system, nsteps, flush, torch):
    """d ln psi/dp and dE_L/dp for every walker folded into the FP64 O/H accumulators (one
    champ_param_grad + champ_accumulate_oh per step; with several ranks also the all-reduce of
    the accumulators); the walkers move by one VMC sweep between steps, outside the timing."""
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
        eng._check(eng.lib.champ_accumulate_oh(eng.h, None, None, None))
        if multi:
            reduce_oh(eng)
        e1.record()
        torch.cuda.synchronize()
        if k >= 2:
            tpg += e0.elapsed_time(e1)
    return tpg


def vmc_arm(system, nw, prec, steps, warmup, flush, torch, rank, world, x0=None, pg_steps=0, clocks=False,
            mover=1):
    from champ_b200.engine import Engine
    eng = Engine(system, nw, prec)
    eng.set_walkers(x0 if x0 is not None else system_walkers(system, nw, seed=1000 + rank))
    if mover != 1:
        eng.set_mover(mover)
    if x0 is None:
        eng.vmc_sweeps(10, SEED + rank, sweep0=0, step=step_size(system), stats=False)  # equilibration
    # launch options that change only the speed (champ_autotune), chosen before the timed region
    tuned = eng.autotune(nsweep=2, seed=SEED + 7, step=step_size(system))
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) if clocks else None
    if clk:
        clk.start()
        time.sleep(0.5)
    tw = time.perf_counter()
    ms, ph = time_sweeps(eng, system, steps, warmup, flush, torch, 100)
    tw = time.perf_counter() - tw
    cl = clk.stop() if clk else None
    ms = allmax(ms)
    out = {"value": nw * world * system.nelec * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps,
           "steps": steps, "precision": prec, "wall_s_timed_region": tw,
           "kernels_ms_per_step": {k: v[0] / steps for k, v in ph.items() if v[1]},
           "launches_per_step": eng.get_option("launches_per_sweep"), "autotune": tuned}
    if cl:
        out["clocks"] = cl
    if pg_steps:
        nj, ncsf, norb = eng.nparam()
        tpg = allmax(time_param_grad(eng, system, pg_steps, flush, torch))
        out["param_grad"] = {"value": nw * world * pg_steps / (tpg * 1e-3), "unit": "param-grad samples/s",
                             "ms_per_step": tpg / pg_steps, "n_params": nj + ncsf + norb,
                             "params": {"jastrow": nj, "csf": ncsf, "orbital": norb}}
    return out, eng


def energy_error(system, x, a="mixed", b="fp64"):
    """|E_L(a) - E_L(b)| per sample on identical walkers (champ_eval_full of both engines)."""
    from champ_b200.engine import Engine
    nw = x.shape[0]
    ea, eb = Engine(system, nw, a), Engine(system, nw, b)
    ea.set_walkers(x)
    eb.set_walkers(x)
    ra, rb = ea.eval_full(), eb.eval_full()
    sd = ra["energy"] - rb["energy"]
    d = np.abs(sd)
    ea.close()
    eb.close()
    return {"walkers": nw, "max_abs_dEL_Ha": float(d.max()), "median_abs_dEL_Ha": float(np.median(d)),
            "frac_samples_within_1e-6_Ha": float(np.mean(d <= 1e-6)), "mean_dEL_Ha": float(sd.mean()),
            "mean_dEL_stderr_Ha": float(sd.std() / np.sqrt(nw))}


def roofline_for(system, nw, arm, clocks, prec):
    """Compute roofline of the dominant kernel of the arm's sweep: counted FLOPs per walker x
    walkers / the kernel's device time per launch, against the CUDA-core FMA rate of its
    precision at the measured SM clock."""
    ks = arm["kernels_ms_per_step"]
    if not ks:
        return None
    kern = max(ks, key=ks.get)
    kprec = {"moves": "fp64" if prec == "fp64" else "fp32", "eval": "fp64",
             "sweep": "fp64" if prec == "fp64" else "fp32"}[kern]
    key = (system.name, kern, kprec)
    mhz = (clocks or {}).get("sm_mhz") or measured_peaks()[0].get("sm_max_mhz", 1965.0)
    peak = 2 * NSM * FMA_PER_SM_CLK[kprec] * mhz * 1e6 / 1e12
    fpw, dpw = FLOPS_PER_WALKER.get(key), DRAM_PER_WALKER.get(key)
    t = ks[kern] * 1e-3
    name = {"eval": "FP64 full evaluation (k_el_jas, k_el_orb, k_el_inv, k_el_fin)", "moves": "k_vmc<float> move phase",
            "sweep": "k_vmc (fused sweep)"}[kern]
    out = {"bound": f"{kprec} FMA rate (CUDA cores; FP64 tensor cores run at the same rate)", "kernel": name,
           "unit": "TFLOP/s", "peak": peak,
           "peak_source": f"{FMA_PER_SM_CLK[kprec]} {kprec.upper()} FMA/clk/SM x {NSM} SMs x 2 x {mhz:.0f} MHz (median "
                          f"SM clock measured in the timed region)",
           "share_of_step": ks[kern] / arm["ms_per_step"], "kernel_ms": ks[kern]}
    if fpw:
        out["achieved"] = fpw * nw / t / 1e12
        out["frac"] = out["achieved"] / peak
        out["flops_per_walker"] = fpw
    else:
        out["achieved"] = None
        out["frac"] = None
        out["note"] = "FLOPs per walker not yet counted for this kernel"
    out["traffic"] = dpw * nw if dpw else None
    if dpw:
        hbm = measured_peaks()[0]["hbm_gbs"]
        out["dram_gbs"] = dpw * nw / t / 1e9
        out["dram_frac_of_measured_hbm"] = out["dram_gbs"] / hbm
    return out


def measure_dmc(system, target, nstep, torch, prec):
    """DMC (system 4): drift-diffusion moves (gradients before and after each proposal), E_L,
    reweighting and branching of the whole population per step, pairs of steps replayed as CUDA
    graphs; e-moves/s = sum over steps of population x electrons / device time."""
    from champ_b200.engine import Engine
    eng = Engine(system, int(1.6 * target), prec)
    eng.set_walkers(system_walkers(system, target, seed=11))
    eng.vmc_sweeps(20, SEED, sweep0=0, step=step_size(system), stats=False)
    eng.dmc_init(target, 0.01)
    eng.dmc_steps(250, seed=SEED)  # equilibration (the population settles within about 250 steps), graph capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    st = eng.dmc_steps(nstep, seed=SEED + 1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    moves = float(st[:, 0].sum()) * system.nelec
    eng.close()
    e_step = st[:, 2] / st[:, 1]
    nb = 10
    blocks = e_step[: len(e_step) // nb * nb].reshape(nb, -1).mean(axis=1)
    return {"workload": f"{system.name}: DMC, target population {target}, tau 0.01", "precision": prec,
            "value": moves / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / nstep, "steps": nstep,
            "population": [float(st[:, 0].min()), float(st[:, 0].mean()), float(st[:, 0].max())],
            "energy_Ha": float(e_step.mean()), "energy_err_Ha": float(blocks.std(ddof=1) / np.sqrt(nb)),
            "step": "per walker: N drift-diffusion proposals (gradient before and after), Green's-function "
                    "acceptance, updates; E_L with NLPP; reweighting; branching; one CUDA graph per two steps",
            "note": "the timed call includes one device-to-host copy of the step statistics and population"}


def e2e_of(eng, system, nw, nsteps, world, torch):
    """End to end through champ_vmc_run_host: walkers from pinned host memory, state rebuild, one
    sweep, E_L and walkers back to pinned host memory, every step."""
    import ctypes as C
    xh = torch.empty((nw, system.nelec, 3), dtype=torch.float64, pin_memory=True)
    xh.copy_(torch.from_numpy(eng.get_walkers()))
    elh = torch.empty((nw,), dtype=torch.float64, pin_memory=True)
    px = C.cast(xh.data_ptr(), C.POINTER(C.c_double))
    pel = C.cast(elh.data_ptr(), C.POINTER(C.c_double))
    for i in range(2):
        eng._check(eng.lib.champ_vmc_run_host(eng.h, nw, px, 1, SEED, 20000 + i, step_size(system), pel))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(nsteps):
        eng._check(eng.lib.champ_vmc_run_host(eng.h, nw, px, 1, SEED, 20010 + k, step_size(system), pel))
    te = allmax(time.perf_counter() - t0)
    return {"value": nw * world * system.nelec * nsteps / te, "unit": UNIT,
            "h2d_bytes_per_step": nw * system.nelec * 3 * 8, "d2h_bytes_per_step": nw * system.nelec * 3 * 8 + nw * 8,
            "call": "champ_vmc_run_host (walkers host->device, FP64 state rebuild without E_L (inverse, log-det, move tables), 1 sweep, E_L and walkers device->host)"}


def main():
    global ARGS
    args = ARGS = parse()
    from champ_b200 import system as S
    system = S.get_system(args.system)
    rank, world, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, system, rank, world)
        return
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    nw = args.walkers or system.walkers
    prec = args.precision
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    pg_steps = max(3, args.steps // 5)
    head, eng = vmc_arm(system, nw, prec, args.steps, args.warmup, flush, torch, rank, world,
                        pg_steps=0 if args.quick else pg_steps, clocks=True)
    xw = eng.get_walkers()
    e2e = e2e_of(eng, system, nw, max(3, args.steps // 4), world, torch)
    eng.close()
    arms = {}
    if not args.quick:
        for p2 in ("fp64", "fp32"):
            if p2 == prec:
                continue
            a, e2 = vmc_arm(system, nw, p2, max(3, args.steps // 2), 2, flush, torch, rank, world, x0=xw,
                            pg_steps=max(2, pg_steps // 2) if p2 == "fp64" else 0)
            e2.close()
            arms[p2] = a
        # the reference's default mover (accelerated Metropolis, imetro 6): drift before and after
        # each proposal, so more work per move than the Gaussian steps of the headline
        a6, e6 = vmc_arm(system, nw, prec, max(3, args.steps // 2), 2, flush, torch, rank, world, x0=xw, mover=6)
        e6.close()
        arms[f"{prec}_imetro6"] = {k: a6[k] for k in ("value", "unit", "ms_per_step", "kernels_ms_per_step")}
        if prec == "mixed":
            arms["mixed_over_fp64"] = {"e-moves/s": head["value"] / arms["fp64"]["value"],
                                       "param-grad samples/s": head["param_grad"]["value"] /
                                       arms["fp64"]["param_grad"]["value"]}
    err = energy_error(system, xw[: min(nw, 1024)], prec, "fp64") if prec != "fp64" else None
    fp32_err = energy_error(system, xw[: min(nw, 1024)], "fp32", "fp64") if not args.quick else None
    roof = roofline_for(system, nw, head, head.get("clocks"), prec)
    others = {}
    if not args.quick and world == 1:
        # the other benchmark systems: e-moves/s mixed and FP64 (systems 1, 2), param-grad samples/s
        # at 16384 walkers with ~500 parameters (system 3), DMC (system 4)
        for k in (1, 2):
            sk = S.get_system(k)
            a, e1 = vmc_arm(sk, sk.walkers, "mixed", max(5, args.steps), 3, flush, torch, rank, world,
                            pg_steps=3 if k == 2 else 0)
            x1 = e1.get_walkers()
            e1.close()
            b, e2 = vmc_arm(sk, sk.walkers, "fp64", max(5, args.steps), 3, flush, torch, rank, world, x0=x1,
                            pg_steps=3 if k == 2 else 0)
            e2.close()
            others[f"system{k}"] = {"workload": config_of(sk, sk.walkers, "mixed")["workload"],
                                    "walkers": sk.walkers, "mixed": a, "fp64": b,
                                    "mixed_error": energy_error(sk, x1[:1024])}
            if rank == 0 and not args.no_cpu_baseline:
                others[f"system{k}"]["cpu_baseline"] = cpu_sample(sk, 5.0)
        s3 = S.get_system(3)
        a3, e3 = vmc_arm(s3, s3.walkers, "mixed", 3, 2, flush, torch, rank, world, pg_steps=3)
        x3 = e3.get_walkers()
        e3.close()
        b3, e3 = vmc_arm(s3, s3.walkers, "fp64", 3, 2, flush, torch, rank, world, x0=x3, pg_steps=3)
        e3.close()
        others["system3"] = {"workload": config_of(s3, s3.walkers, "mixed")["workload"], "walkers": s3.walkers,
                             "param_grad_mixed": a3["param_grad"], "param_grad_fp64": b3["param_grad"],
                             "vmc_mixed": {k: a3[k] for k in ("value", "ms_per_step")},
                             "vmc_fp64": {k: b3[k] for k in ("value", "ms_per_step")}}
        s4 = S.get_system(4)
        others["system4_dmc"] = {"mixed": measure_dmc(s4, s4.walkers, max(20, args.steps), torch, "mixed"),
                                 "fp64": measure_dmc(s4, s4.walkers, max(20, args.steps), torch, "fp64")}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.quick:
        cpu = cpu_sample(system, 12.0)
    if rank == 0:
        launches = head["launches_per_step"] * args.steps
        line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": {"mixed": "f32 moves + f64 E_L", "fp64": "f64", "fp32": "f32+f64"}[prec],
                "data": "synthetic", "config": dict(config_of(system, nw, prec), autotune=head.get("autotune")),
                "clocks": head.get("clocks"),
                "gpu_launches": launches, "kernels_ms_per_step": head["kernels_ms_per_step"],
                "roofline": roof, "param_grad": head.get("param_grad"), "mixed_error": err,
                "arms": arms, "fp32_error": fp32_err, "e2e": e2e, "cpu_baseline": cpu,
                "wall_s_timed_region": head["wall_s_timed_region"], "other_systems": others}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
