"""Work split across GPUs, one process per GPU (torch.distributed: NCCL
between GPUs, gloo on CPU).

* Batches of independent integrals (integrate_sharded): the batch is cut
  into contiguous shards, one per rank, and each rank integrates its shard
  on its own device with no communication on the data path.  One gather of
  fixed-size result records at the end gives every rank the full list.
* Batches of uneven difficulty (integrate_balanced,
  integrate_batch_balanced): the integrals are dealt to the ranks by a
  greedy longest-first split of estimated costs -- the region counts of a
  cheap probe at a looser tolerance, each rank probing a contiguous shard
  and one gather sharing the counts -- so that the ranks finish together.
* One integral (integrate_split): the reference's own multi-device split
  (GPUquad.h:430-609, GPUKernelquad.cu:729-906).  Every rank runs the same
  breadth-first first phase (deterministic, so the ranks agree on the
  leftover boxes without exchanging them), refines a contiguous share of
  the leftover boxes depth-first (the reference's cut,
  GPUKernelquad.cu:759-768), and one all-reduce of a few FP64 numbers --
  value, error, regions, evaluations, failed boxes, non-finite flag --
  combines the shares.  The reference's final status test follows
  (GPUquad.h:713).

Failures are collective: a rank whose shard raises still joins the gather
with an error mark, and every rank then raises, so no rank waits on a peer
that has given up.
"""
from __future__ import annotations

from typing import Callable, Sequence

import torch
import torch.distributed as dist

from . import CubatureError, ERR_INVALID, Result

_FIELDS = ("integral", "error", "nregions", "neval", "status", "iterations", "state")


def shard_bounds(count: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous shard [start, stop) of `count` items for `rank` of `world`;
    shard sizes differ by at most one, the larger ones first."""
    if world <= 0 or not 0 <= rank < world or count < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _pack(results: Sequence[Result], rows: int, failed: bool, device) -> torch.Tensor:
    t = torch.zeros(rows, len(_FIELDS) + 2, dtype=torch.float64, device=device)
    for i, r in enumerate(results):
        t[i, : len(_FIELDS)] = torch.tensor([float(getattr(r, k)) for k in _FIELDS],
                                            dtype=torch.float64)
        t[i, -2] = 1.0  # row holds a result
    t[:, -1] = 1.0 if failed else 0.0
    return t


def _unpack(row) -> Result:
    v = [float(x) for x in row[: len(_FIELDS)]]
    return Result(integral=v[0], error=v[1], nregions=int(v[2]), neval=int(v[3]),
                  status=int(v[4]), iterations=int(v[5]), state=int(v[6]))


def integrate_sharded(integrate: Callable[[int, int], Sequence[Result]], count: int,
                      group=None) -> list[Result]:
    """Run integrate(start, stop) on this rank's shard of `count` integrals
    and return the results of all ranks, in order, on every rank.

    `integrate` maps a shard to its results (for the GPU engine:
    ``lambda a, b: ctx.integrate_batch(fam, n, params[a:b], ...)``).  Without
    an initialised process group this is a plain call on the whole range."""
    if not (dist.is_available() and dist.is_initialized()):
        return list(integrate(0, count))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    start, stop = shard_bounds(count, world, rank)
    rows = max(1, shard_bounds(count, world, 0)[1])  # the largest shard
    failed, message = False, ""
    try:
        local = list(integrate(start, stop)) if stop > start else []
        if len(local) != stop - start:
            raise CubatureError(ERR_INVALID, "shard returned the wrong number of results")
    except Exception as exc:  # every rank must still reach the gather
        failed, message, local = True, f"rank {rank}: {exc}", []
    device = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    mine = _pack(local, rows, failed, device)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    bad = [r for r in range(world) if float(parts[r][0, -1]) != 0.0]
    if bad:
        raise CubatureError(ERR_INVALID, message or f"integration failed on rank(s) {bad}")
    out: list[Result] = []
    for r in range(world):
        a, b = shard_bounds(count, world, r)
        host = parts[r].cpu()
        out.extend(_unpack(host[i]) for i in range(b - a))
    return out


def balanced_assignment(costs: Sequence[float], world: int) -> list[list[int]]:
    """Greedy longest-first split of items with the given costs over `world`
    ranks: items in decreasing cost (ties by index) each go to the rank with
    the least total so far (ties to the lowest rank).  Each rank's indices
    come back in increasing order.  Deterministic, so every rank computes
    the same split from the same costs."""
    if world <= 0:
        raise ValueError("bad world size")
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


def _gather_rows(local: Sequence[Result], rows: int, failed: bool, message: str, world: int,
                 group):
    device = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    mine = _pack(local, rows, failed, device)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    bad = [r for r in range(world) if float(parts[r][0, -1]) != 0.0]
    if bad:
        raise CubatureError(ERR_INVALID, message or f"integration failed on rank(s) {bad}")
    return [p.cpu() for p in parts]


def integrate_balanced(integrate: Callable[[list[int]], Sequence[Result]],
                       costs: Sequence[float], group=None) -> list[Result]:
    """Run integrate(indices) on this rank's share of the batch, the share
    chosen by balanced_assignment(costs, world), and return the results of
    all ranks in batch order on every rank (one gather).  Without an
    initialised process group this is a plain call on every index."""
    count = len(costs)
    if not (dist.is_available() and dist.is_initialized()):
        return list(integrate(list(range(count))))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shares = balanced_assignment(costs, world)
    rows = max(1, max(len(sh) for sh in shares))
    failed, message = False, ""
    try:
        local = list(integrate(shares[rank])) if shares[rank] else []
        if len(local) != len(shares[rank]):
            raise CubatureError(ERR_INVALID, "share returned the wrong number of results")
    except Exception as exc:  # every rank must still reach the gather
        failed, message, local = True, f"rank {rank}: {exc}", []
    parts = _gather_rows(local, rows, failed, message, world, group)
    out: list[Result | None] = [None] * count
    for r in range(world):
        for i, idx in enumerate(shares[r]):
            out[idx] = _unpack(parts[r][i])
    return out  # type: ignore[return-value]


def probe_costs(ctx, family, ndim: int, params: Sequence, epsrel: float, epsabs: float,
                opts=None, factor: float = 100.0, group=None) -> list[float]:
    """Estimated cost of each integral of a batch: its region count at
    epsrel * factor (a run a small fraction of the real one's cost).  Each
    rank probes a contiguous shard; one gather gives every rank all counts."""
    loose = min(0.5, epsrel * factor)

    def run(a: int, b: int):
        return ctx.integrate_batch(family, ndim, list(params)[a:b], loose, epsabs, opts)

    return [float(r.nregions) for r in integrate_sharded(run, len(params), group)]


def integrate_batch_balanced(ctx, family, ndim: int, params: Sequence, epsrel, epsabs,
                             opts=None, group=None, costs: Sequence[float] | None = None
                             ) -> list[Result]:
    """ctx.integrate_batch over all ranks with a difficulty-balanced split
    (probe_costs when no costs are given); scalar tolerances."""
    if costs is None:
        costs = probe_costs(ctx, family, ndim, params, epsrel, epsabs, opts, group=group)
    plist = list(params)

    def run(idx: list[int]):
        return ctx.integrate_batch(family, ndim, [plist[i] for i in idx], epsrel, epsabs, opts)

    return integrate_balanced(run, costs, group)


_NONFINITE = 1 << 30


def integrate_split(shard: Callable[[int, int], tuple], epsrel: float, epsabs: float,
                    group=None) -> Result:
    """One integral with its second phase split over the ranks.

    shard(rank, world) runs the first phase and this rank's share of the
    leftover boxes and returns (phase1, part): the first phase's result
    (finished sums, or the converged result when no box was left) and the
    share's value, error, regions and evaluations with its failed-box count
    in `status` (or the non-finite status).  Every rank returns the same
    combined Result.  Without a process group this is the world-1 case."""
    if dist.is_available() and dist.is_initialized():
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    else:
        world, rank, group = 1, 0, None
    failed, message = 0.0, ""
    p1 = part = None
    try:
        p1, part = shard(rank, world)
    except Exception as exc:  # every rank must still reach the all-reduce
        failed, message = 1.0, f"rank {rank}: {exc}"
    if part is not None:
        nonfin = 1.0 if part.status == _NONFINITE else 0.0
        fail_boxes = 0.0 if part.status == _NONFINITE else float(part.status)
        vec = [part.integral, part.error, float(part.nregions), float(part.neval), fail_boxes,
               nonfin, failed]
    else:
        vec = [0.0] * 6 + [failed]
    if world > 1:
        device = torch.device("cuda", torch.cuda.current_device()) \
            if dist.get_backend(group) == "nccl" else torch.device("cpu")
        t = torch.tensor(vec, dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        vec = [float(x) for x in t.cpu()]
    if vec[6] != 0.0:
        raise CubatureError(ERR_INVALID, message or "integration failed on another rank")
    value = p1.integral + vec[0]
    error = p1.error + vec[1]
    nonfinite = vec[5] != 0.0 or p1.status == _NONFINITE
    status = int(vec[4])
    if error <= max(epsrel * abs(value), epsabs):
        status = 0
    if nonfinite:
        status = _NONFINITE
    return Result(integral=value, error=error, nregions=p1.nregions + int(vec[2]),
                  neval=p1.neval + int(vec[3]), status=status, iterations=p1.iterations,
                  state=1)


def integrate_split_engine(ctx, f, epsrel: float, epsabs: float, opts=None,
                           group=None) -> Result:
    """integrate_split with this rank's GPU engine (ctx.integrate_shard)."""
    return integrate_split(lambda r, w: ctx.integrate_shard(f, epsrel, epsabs, r, w, opts),
                           epsrel, epsabs, group)


def integrate_batch_sharded(ctx, family, ndim: int, params: Sequence, epsrel, epsabs,
                            opts=None, group=None) -> list[Result]:
    """ctx.integrate_batch over all ranks: each rank integrates its shard of
    `params` on its own device (ctx is this rank's context)."""
    def run(a: int, b: int):
        er = epsrel if isinstance(epsrel, (int, float)) else list(epsrel)[a:b]
        ea = epsabs if isinstance(epsabs, (int, float)) else list(epsabs)[a:b]
        return ctx.integrate_batch(family, ndim, list(params)[a:b], er, ea, opts)

    return integrate_sharded(run, len(params), group)
