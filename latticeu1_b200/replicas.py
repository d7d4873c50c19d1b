"""Independent Markov chains across ranks (one process per GPU).

The U(1) update has no exchange between chains, so multi-GPU runs are
replicas: rank r evolves its own lattice with the same seed and chain
number r folded into every Philox counter (disjoint random streams by
construction).  The only cross-rank traffic is reporting: the max of the
ranks' device times and a gather of per-chain observables, both through
torch.distributed (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os

import torch
import torch.distributed as dist


def world() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def chain_id(rank: int, chains_per_rank: int = 1, index: int = 0) -> int:
    """Philox chain number of chain `index` on `rank` (unique over the job)."""
    c = rank * chains_per_rank + index
    if not 0 <= c < 65536:
        raise ValueError("at most 65536 chains")
    return c


def _device() -> torch.device:
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Max of a per-rank scalar (e.g. device milliseconds of the timed region)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_observables(values: list[float]) -> list[list[float]]:
    """All ranks' per-chain observable vectors (same length on every rank)."""
    if not (dist.is_available() and dist.is_initialized()):
        return [list(map(float, values))]
    t = torch.tensor(values, dtype=torch.float64, device=_device())
    out = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [o.cpu().tolist() for o in out]
