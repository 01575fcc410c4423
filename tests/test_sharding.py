"""Event sharding across ranks (the multi-GPU path: independent events,
host-side collectives only), exercised with two gloo ranks on the CPU."""
import json
import multiprocessing as mp
import socket

import pytest

import numpy as np

import shard_worker
import slab_worker
from vhlle_b200.sharding import halo_plan, shard_events, slab_grid, slab_ranges


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


@pytest.mark.parametrize("nz,world", [(51, 2), (101, 8), (21, 3), (12, 2)])
def test_slab_ranges_and_halo_plans_match(nz, world):
    r = slab_ranges(nz, world)
    assert r[0][0] == 0 and r[-1][1] == nz
    plans = [halo_plan(r, k) for k in range(world)]
    for k in range(world):
        a, b, c, d = r[k]
        assert a < b and c <= a and d >= b
        if k:
            assert r[k - 1][1] == a and a - c == min(6, a)
        for peer, zs, ns, zr, nr in plans[k]:
            # what k sends is owned by k and is what its peer receives into
            # its halo, plane for plane in global coordinates
            assert a <= c + zs and c + zs + ns <= b
            back = [p for p in plans[peer] if p[0] == k][0]
            assert back[4] == ns and r[peer][2] + back[3] == c + zs
            assert not (a <= c + zr < b) and nr == back[2]


def test_slab_ranges_reject_slabs_thinner_than_a_halo():
    with pytest.raises(ValueError):
        slab_ranges(11, 2)


def test_slab_grids_keep_the_cell_size_bit_for_bit():
    from vhlle_b200 import workloads as W
    for s in (W.glauber3d_setup(11, 11, 51), W.large_event_setup(0, 11, 11, 101), W.small_glauber3d(9, 25)):
        g = s.grid
        for a, b, c, d in slab_ranges(g.nz, 4):
            sg = slab_grid(g, c, d)
            assert sg.dz == g.dz and sg.nz == d - c and sg.etamin == g.etamin + c * g.dz


def test_two_gloo_ranks_slab_decomposed_event_equals_whole_grid(tmp_path):
    """One event split along eta between two gloo ranks, 6 halo planes
    exchanged once per step: after 6 steps every owned plane of every field
    is bit-identical to the whole grid evolved in one process (oracle)."""
    import pyoracle as P
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=slab_worker.run, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    z = np.load(tmp_path / "slabs.npz")
    setup = slab_worker.event()
    o = P.OracleRun(setup)
    assert o.step(6) == 0
    g = setup.grid
    assert float(z["tau"]) == o.tau_now
    for k in slab_worker.FIELDS:
        want = o.state[k].reshape(slab_worker.NCOMP[k], g.nz, g.nx * g.ny)
        assert np.array_equal(z[k], want, equal_nan=True), k


def test_merge_slab_surfaces_restores_the_cube_order():
    """Elements of two slabs (iz 2-4 and 5-7), each in its own cube order,
    merge into the whole grid's order: (ix, iy, iz) with iz fastest, a
    cube's elements in their order."""
    import numpy as np
    from vhlle_b200 import sharding as S
    whole = []
    for ix in (2, 3):
        for iy in (2, 3):
            for iz in range(2, 8):
                for k in range(1 + (ix + iy + iz) % 3):  # 1-3 elements per cube
                    whole.append((ix, iy, iz, k))
    whole = np.array(whole)
    rec = np.zeros((len(whole), 29))
    rec[:, 0] = np.arange(len(whole))  # the whole grid's element index
    parts = []
    for lo, hi in ((2, 5), (5, 8)):
        sel = (whole[:, 2] >= lo) & (whole[:, 2] < hi)
        parts.append((rec[sel], whole[sel, :3].astype(np.int32)))
    merged = S.merge_slab_surfaces(parts)
    assert np.array_equal(merged[:, 0], np.arange(len(whole)))
    t = S.merge_slab_totals([{"E": 1.0, "S": 2.0}, {"E": 0.5, "S": 1.0}])
    assert t == {"E": 1.5, "S": 3.0}


def test_slab_window_covers_the_owned_planes():
    from vhlle_b200 import sharding as S
    ranges = S.slab_ranges(41, 3)
    got = [S.slab_window(ranges, r, 41) for r in range(3)]
    for (a, b, c, d), (o0, o1, z0, nz) in zip(ranges, got):
        assert (o0 + z0, o1 + z0, nz) == (a, b, 41) and o1 <= d - c
