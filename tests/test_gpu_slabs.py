"""One event split along eta into slab contexts (the multi-GPU layout of a
single large event, vhlle_b200.sharding), here all on one GPU: every slab
steps on its own, then the halo planes go from owner to neighbour through
vh_pack_planes / vh_unpack_planes and a device buffer (between GPUs, NCCL
send/recv of the same buffers).  After every step each slab's owned planes
hold the whole grid's values bit for bit."""
import numpy as np
import pytest

from vhlle_b200 import capi
from vhlle_b200 import sharding as S
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu

NCOMP = dict(Q=7, Qh=7, Qprev=7, pi=10, piH=10, Pi=1, PiH=1, m=3, viscCorrCut=1)


def _exchange(hs, ranges, nxy, torch):
    for r, h in enumerate(hs):
        for peer, zs, ns, _, _ in S.halo_plan(ranges, r):
            back = [p for p in S.halo_plan(ranges, peer) if p[0] == r][0]
            assert back[4] == ns
            buf = torch.empty(capi.VH_PLANE_DOUBLES * ns * nxy, dtype=torch.float64, device="cuda")
            h.pack_planes(zs, ns, buf.data_ptr())
            hs[peer].unpack_planes(back[3], ns, buf.data_ptr())
    for h in hs:
        h.sync()


@pytest.mark.parametrize("case", [
    ("glauber_101x101x51_2slabs", lambda: W.glauber3d_setup(), 2, 12),
    ("large_nb_61x61x41_3slabs", lambda: W.large_event_setup(0, 61, 61, 41, eos=W.nb_table(200, 20)),
     3, 10),
], ids=lambda c: c[0])
def test_gpu_slabs_equal_the_whole_grid(case):
    torch = pytest.importorskip("torch")
    _, fac, nslabs, nsteps = case
    setup = fac()
    g = setup.grid
    nxy = g.nx * g.ny
    ranges = S.slab_ranges(g.nz, nslabs)
    hs = [capi.GpuHydro(S.slab_setup(setup, c, d)) for a, b, c, d in ranges]
    whole = capi.GpuHydro(setup)
    for step in range(nsteps):
        for h in hs:
            h.step(1)
        whole.step(1)
        _exchange(hs, ranges, nxy, torch)
        if step in (0, nsteps - 1):
            want = whole.get_state()
            for (a, b, c, d), h in zip(ranges, hs):
                got = h.get_state()
                for k, n in NCOMP.items():
                    w = want[k].reshape(n, g.nz, nxy)[:, a:b]
                    v = got[k].reshape(n, d - c, nxy)[:, a - c:b - c]
                    assert np.array_equal(v, w, equal_nan=True), (step, k, a, b)
    assert all(h.tau == whole.tau for h in hs)
    for h in hs + [whole]:
        h.close()


@pytest.mark.parametrize("nslabs", [2, 3])
def test_gpu_slab_surfaces_and_totals_equal_the_whole_grid(nslabs):
    """Each slab's freeze-out output of its owned planes (vh_set_slab): the
    corona at tau0 and the surface after the steps, merged in the order of
    the elements' hypercubes (sharding.merge_slab_surfaces), are the whole
    grid's elements in its order, within the record tolerance (a slab's eta
    coordinates start from its own first plane); nsusp adds up exactly and
    the totals within 1e-10 (1e-12 of E for the sums that cancel)."""
    torch = pytest.importorskip("torch")
    from test_gpu_surface import rec_close_scaled
    setup = W.glauber3d_setup(61, 61, 41)
    g = setup.grid
    nxy = g.nx * g.ny
    ranges = S.slab_ranges(g.nz, nslabs)
    hs = [capi.GpuHydro(S.slab_setup(setup, c, d)) for a, b, c, d in ranges]
    for r, h in enumerate(hs):
        h.set_slab(*S.slab_window(ranges, r, g.nz))
    whole = capi.GpuHydro(setup)

    def check(kind):
        if kind == "corona":
            rw, iw = whole.corona()
            parts = [(h.corona()[0], h.surface_cells()) for h in hs]
        else:
            rw, iw = whole.surface()
            parts = []
            nsusp = 0
            for h in hs:
                r, info = h.surface()
                parts.append((r, h.surface_cells()))
                nsusp += info["nsusp"]
            assert nsusp == iw["nsusp"]
        rm = S.merge_slab_surfaces(parts)
        assert rm.shape == rw.shape and len(rw) > 100, (kind, rm.shape, rw.shape)
        ok = rec_close_scaled(rm, rw)
        assert ok.all(), (kind, np.argwhere(~ok)[:5])
        tw = whole.totals()
        ts = S.merge_slab_totals([h.totals() for h in hs])
        for k, v in tw.items():
            assert abs(ts[k] - v) <= 1e-10 * abs(v) + 1e-12 * abs(tw["E"]), (kind, k, ts[k], v)

    check("corona")
    for step in range(8):
        for h in hs:
            h.step(1)
        whole.step(1)
        _exchange(hs, ranges, nxy, torch)
    check("surface")
    for h in hs + [whole]:
        h.close()
