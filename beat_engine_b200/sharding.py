"""Frequency sweeps across GPUs: one process per GPU, each with its own
context, a cost-balanced share of the frequency list, and a host-side gather of
the results in the original order.

Every frequency is independent (its own assembly, factorisation, solve and
field), so no data-path collective is involved: the only communication is the
final gather of host results, over whatever process group the caller set up
(NCCL across GPUs, gloo on the CPU).  The gather keeps each result paired with
its frequency index and raises on a missing or duplicated index, the invariant
the reference's sweep asserts between its producer and consumer
(take_sweep_assembly!, src/BeatEngineCore.jl:1556-1573): a mismatched pairing
would publish one frequency's results under another's label.

Every rank takes the same collective step (one all_gather_object) whether its
share succeeded or raised, so one rank's failure ends the call on every rank
with the same error instead of leaving the others blocked in the gather.
"""
from __future__ import annotations

import heapq
from typing import Any, Callable, Sequence


class ShardError(RuntimeError):
    """A rank's share failed, or the gathered results do not pair up with the
    frequency list; raised on every rank."""


def partition(n_items: int, world: int, cost: Sequence[float] | None = None) -> list[list[int]]:
    """Item indices per rank.  With costs, the largest items go first to the
    least-loaded rank (longest-processing-time); equal costs give a
    round-robin split.  Each rank's list is in increasing index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if n_items < 0:
        raise ValueError("n_items must be >= 0")
    if cost is None:
        return [list(range(r, n_items, world)) for r in range(world)]
    if len(cost) != n_items:
        raise ValueError("cost needs one entry per item")
    heap = [(0.0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(n_items), key=lambda j: (-float(cost[j]), j)):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(cost[i]), r))
    return [sorted(s) for s in shares]


def run_sharded(n_items: int, work: Callable[[list[int]], dict[int, Any]], group=None,
                cost: Sequence[float] | None = None) -> list[Any]:
    """Runs this rank's share through work(indices) -> {index: result} and
    returns every result in index order, on every rank.

    With no process group initialised (or group world size 1) this is
    work(range(n_items)) in order."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        rank, world = 0, 1
    else:
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = partition(n_items, world, cost)[rank]
    try:
        local = ("ok", work(mine))
    except Exception as e:  # reported to every rank after the gather
        local = ("error", f"rank {rank}: {type(e).__name__}: {e}")
    if world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    errors = [msg for status, msg in gathered if status == "error"]
    if errors:
        raise ShardError("; ".join(errors))
    out: list[Any] = [None] * n_items
    seen = [False] * n_items
    for _, results in gathered:
        for index, value in results.items():
            if not (0 <= index < n_items):
                raise ShardError(f"result for index {index} outside the {n_items} items")
            if seen[index]:
                raise ShardError(f"two results for index {index}")
            seen[index] = True
            out[index] = value
    missing = [i for i in range(n_items) if not seen[i]]
    if missing:
        raise ShardError(f"no result for indices {missing[:8]}{'...' if len(missing) > 8 else ''}")
    return out


def sweep_sharded(ctx, k_signed, eta, q, opts=None, dirs=None, group=None, cost=None):
    """A frequency sweep split across the ranks of a process group: q is
    F x R x nfreq (frequency f's Neumann data in q[:, :, f]); each rank solves
    its share with ctx.sweep (its own GPU's context) and every rank returns
    (p: N x R x nfreq, far field: M x R x nfreq or None, diagnostics per
    frequency) in frequency order."""
    import numpy as np

    k_signed = np.ascontiguousarray(k_signed, dtype=np.float64).ravel()
    eta = np.ascontiguousarray(eta, dtype=np.float64).ravel()
    nf = k_signed.size
    q = np.asarray(q, dtype=np.complex128)

    def work(indices):
        if not indices:
            return {}
        idx = np.asarray(indices)
        p, ff, diags = ctx.sweep(k_signed[idx], eta[idx], q[:, :, idx], opts, dirs)
        return {int(i): (p[:, :, j], None if ff is None else ff[:, :, j], diags[j]) for j, i in enumerate(indices)}

    results = run_sharded(nf, work, group, cost)
    p = np.stack([r[0] for r in results], axis=2) if nf else None
    ff = None if dirs is None or not nf else np.stack([r[1] for r in results], axis=2)
    return p, ff, [r[2] for r in results]
