"""Sharding independent integrals across ranks (cubature.parallel), run as
two gloo processes on CPU.  Each rank integrates its shard with the oracle's
two-phase engine (the per-rank integrator is a parameter), so the sharding,
gathering and failure paths are checked without a GPU."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "old-gpuintegration_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from cubature import parallel as P  # noqa: E402


def test_shard_bounds_cover_exactly():
    for count in [0, 1, 5, 7, 64, 4096, 4097]:
        for world in [1, 2, 3, 8]:
            got = [P.shard_bounds(count, world, r) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        P.shard_bounds(4, 2, 2)


def test_without_process_group_runs_whole_range():
    calls = []
    out = P.integrate_sharded(lambda a, b: calls.append((a, b)) or
                              [P.Result(1.0, 0.0, 1, 1, 0, 1, 1)] * (b - a), 3)
    assert calls == [(0, 3)] and len(out) == 3


def _cases(count):
    import numpy as np

    rng = np.random.default_rng(11)
    return [(list(np.exp(rng.uniform(0, np.log(20), 3))), list(rng.uniform(0.1, 0.9, 3)))
            for _ in range(count)]


def _oracle_shard(cases, a, b):
    import oracle as O

    R = O.Rule(3)
    out = []
    for av, uv in cases[a:b]:
        r = R.integrate_reference(O.make_integrand("product_peak", 3, av, uv), 1e-6, 1e-12)
        out.append(P.Result(r["value"], r["error"], r["nregions"], r["neval"], r["status"],
                            r["phase1_iters"], 1))
    return out


# One integral whose first phase leaves boxes for the second (a 512-child
# cap), for the split of its second phase across ranks.
SPLIT_CASE = ("product_peak", 4, [30.0, 40.0, 20.0, 35.0], [0.3, 0.6, 0.5, 0.4], 1e-7, 512)


def _oracle_split_shard(rank, world):
    import oracle as O

    fam, n, a, u, eps, cap = SPLIT_CASE
    p1, part = O.Rule(n).integrate_reference_shard(O.make_integrand(fam, n, a, u), eps, 1e-12,
                                                   rank, world, phase1_cap=cap)
    as_res = lambda d: P.Result(d["value"], d["error"], d["nregions"], d["neval"], d["status"],
                                d["phase1_iters"], 1)
    return as_res(p1), as_res(part)


def _split_worker(rank, world, fail_rank, q):
    fam, n, a, u, eps, cap = SPLIT_CASE

    def shard(r, w):
        if r == fail_rank:
            raise RuntimeError("injected failure")
        return _oracle_split_shard(r, w)

    try:
        res = P.integrate_split(shard, eps, 1e-12)
        q.put((rank, "ok", (res.integral, res.error, res.nregions, res.neval, res.status)))
    except P.CubatureError as exc:
        q.put((rank, "error", str(exc)))


def _worker(rank, world, port, count, fail_rank, q, mode="batch"):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    if mode == "split":
        try:
            _split_worker(rank, world, fail_rank, q)
        finally:
            dist.destroy_process_group()
        return
    try:
        cases = _cases(count)

        def shard(a, b):
            if rank == fail_rank:
                raise RuntimeError("injected failure")
            return _oracle_shard(cases, a, b)

        def share(idx):
            if rank == fail_rank:
                raise RuntimeError("injected failure")
            return [_oracle_shard(cases, i, i + 1)[0] for i in idx]

        try:
            if mode == "balanced":
                # costs: the integrals' region counts at a 100x looser tolerance
                res = P.integrate_balanced(share, _probe_costs(cases))
            else:
                res = P.integrate_sharded(shard, count)
            q.put((rank, "ok", [(r.integral, r.nregions, r.status) for r in res]))
        except P.CubatureError as exc:
            q.put((rank, "error", str(exc)))
    finally:
        dist.destroy_process_group()


def _probe_costs(cases):
    import oracle as O

    R = O.Rule(3)
    return [float(R.integrate_reference(O.make_integrand("product_peak", 3, av, uv), 1e-4,
                                        1e-12)["nregions"]) for av, uv in cases]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world, count, fail_rank=-1, mode="batch"):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, count, fail_rank, q, mode))
             for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out)


@pytest.mark.parametrize("count", [5, 8])
def test_sharded_matches_serial(count):
    """Two ranks, each integrating its shard: every rank gets the full
    result list, identical to integrating the batch in one process."""
    serial = [(r.integral, r.nregions, r.status) for r in _oracle_shard(_cases(count), 0, count)]
    out = _run(2, count)
    assert [o[1] for o in out] == ["ok", "ok"]
    for _, _, res in out:
        assert res == serial


def test_failure_on_one_rank_reaches_all():
    """A shard that raises on rank 1 makes both ranks raise (no rank is left
    waiting in the gather)."""
    out = _run(2, 6, fail_rank=1)
    assert [o[1] for o in out] == ["error", "error"]
    assert all("rank 1" in o[2] or "rank(s) [1]" in o[2] for o in out)


@pytest.mark.parametrize("world", [2, 3])
def test_split_second_phase_matches_one_process(world):
    """One integral, its leftover boxes cut into `world` contiguous shares
    (GPUKernelquad.cu:759-768), each refined by its own rank, one
    all-reduce: every rank gets the single-process result -- the same
    region and evaluation counts and status, the same value and error to
    rounding (the shares are summed in another order)."""
    import oracle as O

    fam, n, a, u, eps, cap = SPLIT_CASE
    ref = O.Rule(n).integrate_reference(O.make_integrand(fam, n, a, u), eps, 1e-12,
                                        phase1_cap=cap)
    assert ref["phase2_regions"] >= world
    out = _run(world, 0, mode="split")
    assert [o[1] for o in out] == ["ok"] * world
    for _, _, (value, error, nreg, neval, status) in out:
        assert nreg == ref["nregions"] and neval == ref["neval"] and status == ref["status"]
        assert abs(value - ref["value"]) <= 1e-12 * abs(ref["value"])
        assert abs(error - ref["error"]) <= 1e-12 * abs(ref["value"])


def test_split_failure_on_one_rank_reaches_all():
    out = _run(2, 0, fail_rank=0, mode="split")
    assert [o[1] for o in out] == ["error", "error"]


def test_split_world_one_is_the_plain_result():
    """Without a process group the split is the world-1 case: the oracle's
    own two-phase result."""
    import oracle as O

    fam, n, a, u, eps, cap = SPLIT_CASE
    ref = O.Rule(n).integrate_reference(O.make_integrand(fam, n, a, u), eps, 1e-12,
                                        phase1_cap=cap)
    res = P.integrate_split(_oracle_split_shard, eps, 1e-12)
    assert (res.nregions, res.neval, res.status) == (ref["nregions"], ref["neval"],
                                                     ref["status"])
    assert res.integral == ref["value"] and res.error == ref["error"]


def test_balanced_assignment_covers_and_balances():
    """The greedy longest-first split deals every item to exactly one rank,
    is the same on every call, keeps each rank's items in batch order, and
    stays within one item's cost of the best balance (the greedy bound);
    on skewed costs it balances far better than contiguous shards."""
    import numpy as np

    rng = np.random.default_rng(3)
    for count, world in [(0, 2), (1, 3), (7, 2), (100, 3), (4096, 8)]:
        costs = list(np.exp(rng.uniform(0, 6, count)))
        sh = P.balanced_assignment(costs, world)
        assert sh == P.balanced_assignment(costs, world)
        flat = sorted(i for s_ in sh for i in s_)
        assert flat == list(range(count))
        assert all(s_ == sorted(s_) for s_ in sh)
        if count:
            loads = [sum(costs[i] for i in s_) for s_ in sh]
            assert max(loads) - min(loads) <= max(costs) + 1e-9
    costs = [100.0] * 4 + [1.0] * 60  # the hard integrals first, as in a sorted batch
    loads_b = [sum(costs[i] for i in s_) for s_ in P.balanced_assignment(costs, 4)]
    loads_c = [sum(costs[a:b]) for a, b in (P.shard_bounds(64, 4, r) for r in range(4))]
    assert max(loads_b) < 0.5 * max(loads_c)
    with pytest.raises(ValueError):
        P.balanced_assignment([1.0], 0)


@pytest.mark.parametrize("world", [2, 3])
def test_balanced_matches_serial(world):
    """Ranks integrating difficulty-balanced shares (probe costs at a looser
    tolerance) return the whole batch, in batch order, identical to one
    process; a failure on one rank reaches every rank."""
    count = 9
    serial = [(r.integral, r.nregions, r.status) for r in _oracle_shard(_cases(count), 0, count)]
    out = _run(world, count, mode="balanced")
    assert [o[1] for o in out] == ["ok"] * world
    for _, _, res in out:
        assert res == serial
    out = _run(world, count, fail_rank=world - 1, mode="balanced")
    assert [o[1] for o in out] == ["error"] * world
