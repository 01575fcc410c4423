"""The con2prim policy knobs: at a tight stopping tolerance the device step
equals the tight oracle (the reference's algorithm with only the tolerance
changed) bit for bit, and the iteration counters count."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
TIGHT = 1e-13


@pytest.mark.parametrize("case", [
    ("glauber_17x17x9", lambda: W.small_glauber3d(17, 9), 6),
    ("gubser_31x31", lambda: W.gubser_setup(nx=31, ny=31), 10),
], ids=lambda c: c[0])
def test_gpu_tight_equals_tight_oracle(case):
    from vhlle_b200.capi import GpuHydro
    name, fac, n = case
    setup = fac()
    o = P.OracleRun(setup, tol=TIGHT)
    d = GpuHydro(setup)
    d.set_con2prim(TIGHT)
    for s in range(n):
        o.step(1)
        d.step(1)
    bad = compare_states(gpu_state_as_oracle(d.get_state()), o.get_state())
    assert not bad, bad
    d.close()


def test_gpu_con2prim_counts_and_tolerance_bounds():
    from vhlle_b200.capi import GpuHydro, VhError
    setup = W.small_glauber3d(17, 9)
    d = GpuHydro(setup)
    d.con2prim_stats(True)
    d.step(2)
    c_ref, it_ref = d.con2prim_stats(True)
    d.set_con2prim(TIGHT)
    d.step(2)
    c_t, it_t = d.con2prim_stats(False)
    assert c_ref > 0 and c_t > 0
    assert it_t / c_t > it_ref / c_ref  # a tighter stop needs more iterations
    with pytest.raises(VhError):
        d.set_con2prim(1e-3)
    d.close()
