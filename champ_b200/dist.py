"""Multi-rank plumbing: one process per GPU, torch.distributed for the reductions.

Walkers are independent Markov chains, so ranks share nothing on the data path: each rank owns
its own walkers (a contiguous shard of the global population, its own random stream) and runs
the engine on them.  The exchange steps of the reference's MPI runs are reductions only:
  * estimator sums (E_L, E_L^2, acceptance) once per block (vmc.f90 block averages),
  * the linear method's O/H accumulators once per optimisation sample (the MPI sums behind the
    dpsi_dpsi / dpsi_deloc / dpsi_dpsi_eloc averages, deriv_mod.f90:683,898,1375),
  * the total DMC weight and population per step (rundmc_mod.f90:357-358).
Every rank must call these in the same order.  With one rank (or no process group) they are
no-ops that return the local values.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def rank_world() -> tuple[int, int]:
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """(first walker, walker count) of this rank's contiguous share of `total` walkers."""
    base, extra = divmod(total, world)
    count = base + (1 if rank < extra else 0)
    return rank * base + min(rank, extra), count


def walker_seed(seed: int, rank: int) -> int:
    """Seed of a rank's walker stream: distinct ranks draw independent chains."""
    return seed + 1_000_003 * rank


def _active() -> bool:
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def sum_(t: torch.Tensor) -> torch.Tensor:
    """In-place sum over ranks (FP64 on the tensor's device)."""
    if _active():
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t


def max_over_ranks(x: float) -> float:
    """Max of a per-rank number (device timings: the job is as slow as its slowest rank)."""
    if not _active():
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_estimators(esum, e2sum, accept, nsweep: int, nelec: int) -> dict:
    """Global VMC block estimators from per-walker sums of this rank's walkers (champ_vmc_sweeps
    statistics): mean E_L, its variance, and the acceptance ratio over all ranks' walkers."""
    loc = torch.tensor([float(sum(esum)), float(sum(e2sum)), float(sum(accept)), float(len(esum))],
                       dtype=torch.float64)
    if _active() and dist.get_backend() == "nccl":
        loc = loc.cuda()
    sum_(loc)
    s, s2, acc, nw = (float(v) for v in loc.cpu())
    n = nw * nsweep
    mean = s / n
    return {"energy": mean, "variance": s2 / n - mean * mean, "accept": acc / (n * nelec), "walkers": int(nw)}


class _DeviceArray:
    """A CUDA array interface over engine-owned device memory (no copy, no ownership)."""

    def __init__(self, ptr: int, shape, dtype: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": dtype, "data": (ptr, False),
                                         "version": 3, "strides": None}


def oh_tensors(engine) -> tuple[torch.Tensor, torch.Tensor]:
    """The engine's device O/H accumulators as torch tensors (views, no copy)."""
    P1 = sum(engine.nparam()) + 1
    s_ptr, h_ptr = engine.oh_buffers()
    S = torch.as_tensor(_DeviceArray(s_ptr, (P1, P1)), device="cuda")
    H = torch.as_tensor(_DeviceArray(h_ptr, (P1, P1)), device="cuda")
    return S, H


def reduce_oh(engine) -> tuple[torch.Tensor, torch.Tensor]:
    """Sum the O/H accumulators of the last champ_accumulate_oh over all ranks, in place on the
    device (one NCCL all-reduce per matrix).  The engine's stream must have finished them."""
    S, H = oh_tensors(engine)
    torch.cuda.synchronize()
    sum_(S)
    sum_(H)
    return S, H


def reduce_oh_host(S, H):
    """Host-array variant (the O/H returned by Engine.accumulate_oh): sums over ranks in FP64."""
    ts, th = torch.from_numpy(S).clone(), torch.from_numpy(H).clone()
    if _active() and dist.get_backend() == "nccl":
        ts, th = ts.cuda(), th.cuda()
    sum_(ts)
    sum_(th)
    return ts.cpu().numpy(), th.cpu().numpy()


def reduce_dmc_step(weight_sum: float, population: int, weighted_energy: float) -> tuple[float, int, float]:
    """Total weight, population and sum of w E_L over all ranks for one DMC step."""
    t = torch.tensor([weight_sum, float(population), weighted_energy], dtype=torch.float64)
    if _active() and dist.get_backend() == "nccl":
        t = t.cuda()
    sum_(t)
    w, n, we = (float(v) for v in t.cpu())
    return w, int(round(n)), we


__all__ = ["rank_world", "shard", "walker_seed", "sum_", "max_over_ranks", "reduce_estimators", "oh_tensors",
           "reduce_oh", "reduce_oh_host", "reduce_dmc_step"]
