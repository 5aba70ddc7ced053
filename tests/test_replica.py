"""The multi-GPU path on CPU: world-size-2 gloo ranks drive replica.Ranks the
way bench.py drives it under torchrun (barrier around the timed region,
max-over-ranks time, whole-job rate from all ranks' units), plus the host
dispatch helpers. The chain itself shards by frame with no collective on the
data path, so the process group only carries this control traffic."""
import multiprocessing as mp
import os
import socket
import sys
import time

import pytest

import replica as R

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rivet-av1_b200")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, mode):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, PKG)
    import replica as Rw
    try:
        ranks = Rw.Ranks(backend="gloo", timeout_s=15)
        if mode == "bench":
            # the bench's shape: units sharded round robin, a barrier on both
            # sides of the timed region, elapsed time maxed over ranks
            units = Rw.shard(11, ranks.rank, ranks.world)
            ranks.barrier()
            t0 = time.perf_counter()
            time.sleep(0.05 * (ranks.rank + 1))  # rank 1 is the slow one
            ranks.barrier()
            ms = 1e3 * (time.perf_counter() - t0)
            ms_max = ranks.max(ms)
            total = ranks.sum(len(units))
            q.put(("ok", ranks.rank, ms, ms_max, total, units, Rw.aggregate_rate(total, ms_max)))
            ranks.close()
        elif mode == "dead_peer":
            if ranks.rank == 1:
                os._exit(0)  # leaves between steps, nothing in flight
            try:
                ranks.max(1.0)
                q.put(("no_error", ranks.rank))
            except Exception as e:  # noqa: BLE001
                q.put(("error", ranks.rank, type(e).__name__))
    except Exception as e:  # noqa: BLE001
        q.put(("exc", rank, repr(e)))


def _run(world, mode, timeout=90):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    deadline = time.time() + timeout
    expected = world if mode == "bench" else 1
    while len(out) < expected and time.time() < deadline:
        try:
            out.append(q.get(timeout=1.0))
        except Exception:  # noqa: BLE001
            if all(not p.is_alive() for p in procs) and q.empty():
                break
    for p in procs:
        p.join(timeout=max(1.0, deadline - time.time()))
        if p.is_alive():
            p.kill()
            p.join()
    return out


def test_two_gloo_ranks_bench_timing():
    out = _run(2, "bench")
    assert len(out) == 2, out
    assert all(o[0] == "ok" for o in out), out
    by_rank = {o[1]: o for o in out}
    # every rank agrees on the max and the total; the max is the slowest rank's
    ms_max = {o[3] for o in out}
    assert len(ms_max) == 1
    assert ms_max.pop() == pytest.approx(max(o[2] for o in out))
    assert {o[4] for o in out} == {11.0}
    # shards are disjoint and cover every unit
    assert sorted(by_rank[0][5] + by_rank[1][5]) == list(range(11))
    assert not set(by_rank[0][5]) & set(by_rank[1][5])
    # the whole-job rate is the same number on both ranks
    assert by_rank[0][6] == pytest.approx(by_rank[1][6])


def test_dead_peer_surfaces_as_error():
    out = _run(2, "dead_peer", timeout=60)
    assert out and out[0][0] == "error", out


def test_single_rank_is_local():
    r = R.Ranks(backend="gloo", env={"RANK": "0", "WORLD_SIZE": "1"})
    assert r.world == 1 and r.dist is None
    assert r.max(3.5) == 3.5 and r.sum(2) == 2.0
    r.close()


def test_shard_and_seeds():
    for world in (1, 2, 3, 8):
        got = sorted(i for rank in range(world) for i in R.shard(64, rank, world))
        assert got == list(range(64))
        sizes = [len(R.shard(64, rank, world)) for rank in range(world)]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        R.shard(4, 2, 2)
    seeds = {R.frame_seed(r, i) for r in range(8) for i in range(64)}
    assert len(seeds) == 8 * 64
    with pytest.raises(ValueError):
        R.frame_seed(0, 1000)


def test_assign_by_free_memory():
    gib = 2**30
    # the serving mix: 2 large, 6 medium, 24 small streams on 2 GPUs
    demands = [3 * gib] * 2 + [gib] * 6 + [gib // 4] * 24
    place = R.assign_by_free_memory(demands, [40 * gib, 40 * gib])
    load = [sum(d for d, g in zip(demands, place) if g == k) for k in range(2)]
    assert abs(load[0] - load[1]) <= gib // 4
    assert place[0] != place[1]  # the two large streams land on different GPUs
    # deterministic
    assert place == R.assign_by_free_memory(demands, [40 * gib, 40 * gib])
    # uneven free memory fills the larger GPU first
    assert R.assign_by_free_memory([gib], [gib, 2 * gib]) == [1]
    with pytest.raises(ValueError):
        R.assign_by_free_memory([5 * gib], [4 * gib, 4 * gib])
    with pytest.raises(ValueError):
        R.aggregate_rate(10, 0)
    assert R.aggregate_rate(2000, 1000.0) == 2000.0
