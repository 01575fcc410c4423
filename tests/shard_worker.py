"""Child process of the two-rank gloo test: evolves its shard of small
events with the oracle and gathers per-event totals to rank 0."""
import json
import os


def events():
    from vhlle_b200 import workloads as W
    return [W.small_glauber3d(13, 7, seed=1), W.small_glauber3d(17, 9, seed=2, b=4.0),
            W.small_glauber3d(15, 7, seed=3), W.small_glauber3d(11, 5, seed=4)]


def evolve(setup, nsteps=2):
    import pyoracle as P
    o = P.OracleRun(setup)
    assert o.step(nsteps) == 0
    t = o.totals()
    return {"E": t["E"], "Nb1": t["Nb1"], "S": t["S"], "tau": o.tau_now}


def run(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from vhlle_b200.sharding import Ranks, shard_events
    ranks = Ranks(timeout_s=60)
    evs = events()
    mine = shard_events([e.grid.ncells for e in evs], world, rank)
    res = {i: evolve(evs[i]) for i in mine}
    ranks.barrier()
    tmax = ranks.max(float(rank + 1))
    tsum = ranks.sum(float(len(mine)))
    got = ranks.gather(res)
    if rank == 0:
        merged = {}
        for r in got:
            merged.update({str(k): v for k, v in r.items()})
        with open(os.path.join(out_dir, "merged.json"), "w") as f:
            json.dump({"results": merged, "max": tmax, "sum": tsum}, f)
    ranks.close()
