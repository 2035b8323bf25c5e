"""Multi-process host logic of the sharded batch and request routing (gloo, world size 2, CPU)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "diplodocustransport.jl_b200"))

from dtb.shard import gather, route, serve_sharded, shard_range  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_items, costs, q, fail_rank):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "diplodocustransport.jl_b200"))
    from dtb.shard import gather as g_, route as r_, shard_range as s_
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected failure before the gather")
        lo, hi = s_(n_items, rank, world)
        mine = list(range(lo, hi))
        ranks = r_(costs, world)
        my_reqs = [k for k, r in enumerate(ranks) if r == rank]
        allv = g_({"rank": rank, "items": mine, "reqs": my_reqs})
        q.put(("ok", rank, allv))
    except Exception as e:  # reported to the parent; the peer's gather then times out
        q.put(("err", rank, repr(e)))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, n_items, costs, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, n_items, costs, q, fail_rank)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=60) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_shard_range_partitions_exactly():
    for n in (0, 1, 5, 256, 1001):
        for w in (1, 2, 3, 8):
            parts = [shard_range(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(w - 1))
            assert max(b - a for a, b in parts) - min(b - a for a, b in parts) <= 1


def test_route_balances_work():
    costs = [500 + 97 * k % 19500 for k in range(200)]
    ranks = route(costs, 4)
    load = [sum(c for c, r in zip(costs, ranks) if r == j) for j in range(4)]
    assert max(load) - min(load) <= max(costs)
    assert route([1, 1, 1], 2, "round_robin") == [0, 1, 0]
    with pytest.raises(ValueError):
        route([1], 0)


def test_two_ranks_cover_every_instance_and_request_once():
    costs = [500 + (37 * k) % 19500 for k in range(120)]
    out = _run(2, 256, costs)
    assert all(o[0] == "ok" for o in out), out
    allv = out[0][2]
    items = sorted(i for v in allv for i in v["items"])
    reqs = sorted(k for v in allv for k in v["reqs"])
    assert items == list(range(256)) and reqs == list(range(120))
    assert out[1][2] == allv  # every rank sees the same gathered view


def test_failed_rank_is_detected_by_the_peer():
    """A rank that raises before the gather: the peer's collective ends with an error after the
    process-group timeout instead of hanging."""
    out = _run(2, 16, [1.0] * 4, fail_rank=1)
    kinds = {o[1]: o[0] for o in out}
    assert kinds[1] == "err" and kinds[0] == "err"


class _FakeServer:
    """Stands in for one GPU's continuous-batching server on the host: a request's record is
    its step count and the rank that served it; `fail` raises inside the share (a failed GPU)."""

    def __init__(self, rank, steps, fail=False):
        self.rank, self.steps, self.fail = rank, steps, fail
        self.seen = []

    def __call__(self, mine):
        if self.fail:
            raise RuntimeError("injected failure while serving")
        self.seen = list(mine)
        return [{"steps": self.steps[k], "served_by": self.rank} for k in mine]


def _serve_worker(rank, world, port, steps, q, fail_rank):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "diplodocustransport.jl_b200"))
    from dtb.shard import route as r_, serve_sharded as ss_
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        fake = _FakeServer(rank, steps, fail=(rank == fail_rank))
        recs = ss_([float(x) for x in steps], rank, world, fake)
        expect = [k for k, r in enumerate(r_([float(x) for x in steps], world)) if r == rank]
        q.put(("ok", rank, {"recs": recs, "seen": fake.seen, "expect": expect}))
    except Exception as e:
        q.put(("err", rank, repr(e)))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run_serve(world, steps, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_serve_worker, args=(r, world, port, steps, q, fail_rank)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=60) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_served_stream_is_routed_served_once_and_gathered():
    """serve_sharded end to end on two ranks: each rank serves exactly its routed share (the
    admit list), and every rank gets every request's record back, in arrival order."""
    steps = [500 + (7919 * k) % 19500 for k in range(64)]
    out = _run_serve(2, steps)
    assert all(o[0] == "ok" for o in out), out
    by_rank = {o[1]: o[2] for o in out}
    for r in (0, 1):
        assert by_rank[r]["seen"] == by_rank[r]["expect"] and by_rank[r]["seen"]
    recs = by_rank[0]["recs"]
    assert recs == by_rank[1]["recs"]
    assert [x["index"] for x in recs] == list(range(64))
    assert all(x["steps"] == steps[x["index"]] and x["served_by"] == x["rank"] for x in recs)
    loads = [sum(x["steps"] for x in recs if x["rank"] == r) for r in (0, 1)]
    assert abs(loads[0] - loads[1]) <= max(steps)


def test_failed_serving_rank_is_detected_by_the_peer():
    """A rank whose server fails raises; the healthy rank's gather ends with an error after the
    process-group timeout instead of hanging."""
    out = _run_serve(2, [1000] * 8, fail_rank=0)
    kinds = {o[1]: o[0] for o in out}
    assert kinds[0] == "err" and kinds[1] == "err"
