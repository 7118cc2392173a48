"""(T) over several GPUs: contiguous tuple shards and one all-reduce.

The reference hands tuples to DDI processes (static ``div_even`` split of the
i>j>k list, ``triples.F90:101``, then the ``ddi_dlbnext`` queue,
``triples.F90:231,265,295``) and sums the per-process v1 and etd with
``ddi_gsumf`` (``triples.F90:307-308``).  Tuples are independent, so here each
rank (one process per GPU, ``torch.distributed``) takes one contiguous shard of
the plan's tuple list with near-equal summed cost -- an i>j>k tuple costs 1,
a degenerate (i,j,j)/(i,i,j) tuple 1/2 (it builds two of the three W GEMMs at
half the K) -- and runs it through ``TriplesPlan.forward(begin, end)``.  The
partial (ets, etd, v1) are then summed with one all-reduce: the only exchange
step.  Inputs are replicated on every rank; nothing reads a peer's memory.

ets = 2 sum t1 v1 is linear in v1, so summing per-shard ets equals the
reference's ets over the summed v1 up to rounding.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np


def tuple_costs(no: int) -> list:
    """Relative W-build cost of each tuple in plan order: C(no,3) i>j>k tuples at 1,
    then the no(no-1) degenerate tuples at 1/2."""
    n_ijk = no * (no - 1) * (no - 2) // 6
    return [1.0] * n_ijk + [0.5] * (no * (no - 1))


def shard_bounds(costs: Sequence[float], nranks: int) -> list:
    """Boundaries b[0..nranks] of contiguous shards with near-equal summed cost.

    Rank r owns tuples [b[r], b[r+1]).  Shards may be empty when there are fewer
    tuples than ranks; every tuple belongs to exactly one shard."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    n = len(costs)
    total = float(sum(costs))
    bounds, acc, r = [0], 0.0, 1
    for t, c in enumerate(costs):
        acc += c
        if r < nranks and acc >= total * r / nranks:
            bounds.append(t + 1)
            r += 1
    while len(bounds) < nranks:
        bounds.append(n)
    bounds.append(n)
    return bounds


def shard_of(no: int, rank: int, world: int) -> Tuple[int, int]:
    """The [begin, end) tuple range of ``rank`` among ``world`` ranks."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    b = shard_bounds(tuple_costs(no), world)
    return b[rank], b[rank + 1]


def _group_info(group):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return None, 0, 1
    return dist, dist.get_rank(group), dist.get_world_size(group)


def sharded_forward(forward: Callable[[int, int], tuple], no: int, nu: int, group=None,
                    want_v1: bool = True, device: Optional[str] = None) -> tuple:
    """Run this rank's shard with ``forward(begin, end) -> (ets, etd, v1)`` and sum
    the partial results over ``group`` with one all-reduce.

    ``forward`` is normally ``TriplesPlan.forward``; its ``v1`` is the flat
    (nu, no) accumulator.  With ``want_v1`` False only the energies are reduced;
    every rank must pass the same value, since it sets the all-reduce length.
    ``device`` is where the all-reduce buffer lives: the rank's GPU for NCCL,
    ``"cpu"`` for gloo (default: chosen from the group's backend).  Every rank
    makes the same single collective call, also when its shard is empty.
    Returns the global (ets, etd, v1) on every rank."""
    import torch
    dist, rank, world = _group_info(group)
    begin, end = shard_of(no, rank, world)
    ets, etd, v1 = forward(begin, end) if end > begin else (0.0, 0.0, None)
    if want_v1 and v1 is None:
        v1 = np.zeros(nu * no)
    if not want_v1:
        v1 = None
    if dist is None:
        return ets, etd, v1
    if device is None:
        device = f"cuda:{torch.cuda.current_device()}" if dist.get_backend(group) == "nccl" else "cpu"
    n = 2 + (no * nu if want_v1 else 0)
    buf = torch.zeros(n, dtype=torch.float64)
    buf[0], buf[1] = float(ets), float(etd)
    if want_v1:
        buf[2:] = torch.from_numpy(np.ascontiguousarray(v1, dtype=np.float64).reshape(-1))
    buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return float(out[0]), float(out[1]), (out[2:].copy() if want_v1 else None)


def sharded_cc_triples(plan, group=None, want_v1: bool = True) -> tuple:
    """(ets, etd, v1) of the system loaded into ``plan`` (a ``TriplesPlan`` whose
    inputs are set on every rank), each rank running its own tuple shard."""
    def fwd(b, e):
        ets, etd, v1 = plan.forward(b, e, want_v1=want_v1)
        return ets, etd, v1
    return sharded_forward(fwd, plan.no, plan.nu, group=group, want_v1=want_v1)
