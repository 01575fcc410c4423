"""Event sharding across ranks (the multi-GPU path: independent events,
host-side collectives only), exercised with two gloo ranks on the CPU."""
import json
import multiprocessing as mp
import socket

import pytest

import shard_worker
from vhlle_b200.sharding import shard_events


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_partition_the_events(world):
    cells = [61 * 61, 121 * 121 * 61, 81 * 81 * 21, 61 * 61 * 11, 101 * 101 * 51, 5, 5, 70000]
    shards = [shard_events(cells, world, r) for r in range(world)]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(cells)))
    for s in shards:
        assert s == sorted(s)
    loads = [sum(cells[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(cells)


def test_shards_reject_bad_rank():
    with pytest.raises(ValueError):
        shard_events([1, 2], 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_equal_one_process(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=shard_worker.run, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    d = json.loads((tmp_path / "merged.json").read_text())
    assert d["max"] == 2.0 and d["sum"] == 4.0
    evs = shard_worker.events()
    assert sorted(d["results"]) == [str(i) for i in range(len(evs))]
    for i, e in enumerate(evs):
        assert d["results"][str(i)] == shard_worker.evolve(e)
