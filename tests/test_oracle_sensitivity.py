"""How far a last-bit difference goes in the reference's algorithm (the
oracle, bit-equal to the compiled reference): two runs of the same event
whose transformPV stops at |dv| < 1e-13 and < 1e-14, both converged to
round-off, agree to round-off for ten steps and then part in the cells
where the pi limiter, the viscCorrCut flag or a vacuum-edge branch switch.
This is why a path that changes a root find's iteration (a learned start
point, the table slope) or a last bit of exp can be held to 1e-8 only over
the first steps, and is compared with this spread after longer runs."""
import numpy as np

import pyoracle as P
from vhlle_b200 import workloads as W


def _rel(x, y):
    scale = np.abs(y).max()
    d = np.abs(x - y) - 1e-12 * scale
    return np.where(d > 0, d / np.maximum(np.maximum(np.abs(x), np.abs(y)), 1e-300), 0.0)


def test_converged_stops_part_after_some_steps():
    s = W.glauber3d_setup(41, 41, 21, etaS=0.12, seed=20263005, b=3.0)
    a, b = P.OracleRun(s, tol=1e-13), P.OracleRun(s, tol=1e-14)
    assert a.step(10) == 0 and b.step(10) == 0
    for k in ("Q", "pi", "Pi"):
        assert _rel(a.state[k], b.state[k]).max() == 0.0, k
    assert a.step(10) == 0 and b.step(10) == 0
    r = _rel(a.state["pi"], b.state["pi"])
    assert r.max() > 1e-8 and (r > 1e-8).mean() < 1e-2
