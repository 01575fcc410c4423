"""Child process of the two-rank slab test: one event split along eta, each
rank evolving its slab with the oracle and exchanging halo planes with its
neighbour through torch.distributed (gloo, host buffers) once per step;
rank 0 gathers the owned planes."""
import os

import numpy as np

FIELDS = ("Q", "Qh", "Qprev", "pi", "piH", "Pi", "PiH", "m", "vcc")
NCOMP = dict(Q=7, Qh=7, Qprev=7, pi=10, piH=10, Pi=1, PiH=1, m=3, vcc=1)


def event():
    from vhlle_b200 import workloads as W
    return W.small_glauber3d(17, 21, seed=5, b=4.0)


def planes_of(state, nz, nxy, z0, n):
    """The [field][component][plane][nx*ny] layout of vh_pack_planes."""
    return np.concatenate([state[k].reshape(NCOMP[k], nz, nxy)[:, z0:z0 + n].reshape(-1)
                           for k in FIELDS])


def put_planes(state, nz, nxy, z0, n, buf):
    off = 0
    for k in FIELDS:
        m = NCOMP[k] * n * nxy
        state[k].reshape(NCOMP[k], nz, nxy)[:, z0:z0 + n] = buf[off:off + m].reshape(NCOMP[k], n, nxy)
        off += m


def run(rank, world, port, out_dir, nsteps=6):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import pyoracle as P
    from vhlle_b200 import sharding as S
    ranks = S.Ranks(timeout_s=60)
    setup = event()
    g = setup.grid
    nxy = g.nx * g.ny
    rng = S.slab_ranges(g.nz, world)
    a, b, c, d = rng[rank]
    o = P.OracleRun(S.slab_setup(setup, c, d))
    nz = d - c

    def pack(z0, n, buf):
        buf.copy_(torch.from_numpy(planes_of(o.state, nz, nxy, z0, n)))

    def unpack(z0, n, buf):
        put_planes(o.state, nz, nxy, z0, n, buf.numpy())

    def new_buffer(n):
        return torch.empty(47 * n * nxy, dtype=torch.float64)

    for _ in range(nsteps):
        assert o.step(1) == 0
        S.exchange_halos(ranks.dist, rng, rank, pack, unpack, new_buffer)
    mine = {k: o.state[k].reshape(NCOMP[k], nz, nxy)[:, a - c:b - c].copy() for k in FIELDS}
    got = ranks.gather((a, b, mine))
    if rank == 0:
        full = {k: np.concatenate([m[k] for _, _, m in sorted(got, key=lambda x: x[0])], axis=1)
                for k in FIELDS}
        np.savez(os.path.join(out_dir, "slabs.npz"), tau=o.tau_now, **full)
    ranks.close()
