"""Comparison helpers shared by the parity tests."""
import numpy as np

# field names of the oracle / fixtures -> C ABI names
ABI_NAME = dict(Q="Q", Qh="Qh", Qprev="Qprev", pi="pi", piH="piH", Pi="Pi", PiH="PiH", m="m",
                vcc="viscCorrCut")


def mismatch(a, b):
    """(number of differing values, max relative difference) for two arrays,
    NaNs in the same places counting as equal."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    n = int((~same).sum())
    if n == 0:
        return 0, 0.0
    d = np.abs(a - b)[~same]
    scale = np.maximum(np.abs(a), np.abs(b))[~same]
    rel = np.where(scale > 0, d / np.where(scale > 0, scale, 1), 0)
    return n, float(np.nanmax(rel))


def compare_states(got, expect, fields=None, rtol=0.0, atol=0.0):
    """Returns {field: (ndiff, maxrel)} for fields whose values differ beyond
    rtol (relative, scaled by the larger magnitude) or atol."""
    bad = {}
    for k in fields or expect.keys():
        a = np.asarray(got[k], dtype=np.float64).reshape(-1)
        b = np.asarray(expect[k], dtype=np.float64).reshape(-1)
        same = (a == b) | (np.isnan(a) & np.isnan(b))
        tol = np.maximum(rtol * np.maximum(np.abs(a), np.abs(b)), atol)
        ok = same | (np.abs(a - b) <= tol)
        if not ok.all():
            bad[k] = mismatch(a, b)
    return bad


def gpu_state_as_oracle(st):
    """C ABI field names -> oracle field names."""
    inv = {v: k for k, v in ABI_NAME.items()}
    return {inv[k]: v for k, v in st.items()}


def transport_variant(kind, par):
    """The large event's physics on a 25x25x13 grid (200 x 20 (e, nb) table)
    with one of the reference's eta/s or zeta/s forms (src/trancoeff.cpp:
    19-90); parameter values chosen so that each form is active (nonzero
    shear or bulk) over the event's temperature range."""
    from vhlle_b200 import workloads as W
    s = W.large_event_setup(0, 25, 25, 13, eos=W.nb_table(200, 20))
    if kind == "zeta":
        s.zetaSparam = par
        if par == 4:
            s.tr = dict(s.tr, zetaS0=0.02, zetaSPeakEpsilon=0.5, zetaSScaleBeta=1.0,
                        zetaSSigmaMinus=0.5, zetaSSigmaPlus=1.0)
    else:
        s.zetaSparam = 0
        s.etaSparam = par
        s.tr = dict(s.tr, etaSMin=0.08, ah=0.3, al=-0.5, aRho=0.05, T0=0.18,
                    etaSEpsilonMin=1.0, etaSShiftMuB=0.1, etaSScaleMuB=0.2)
    return s


TRANSPORT_VARIANTS = [("zeta", 1), ("zeta", 2), ("zeta", 3), ("zeta", 4),
                      ("eta", 1), ("eta", 2), ("eta", 3)]


def transport_inputs(n=100000, seed=1):
    """Random thermodynamic points [n][6] = e, nb, T, muB, s, p spanning
    every branch of the transport forms (T across 0.1 and the zeta/s peaks,
    e across etaSEpsilonMin and zetaSPeakEpsilon, |s| across 1)."""
    rng = np.random.default_rng(seed)
    e = 10 ** rng.uniform(-3, 2.5, n)
    return np.stack([e, rng.uniform(0, 1, n), rng.uniform(0.05, 0.8, n), rng.uniform(0, 0.9, n),
                     10 ** rng.uniform(-2, 3, n), e / 3 * rng.uniform(0.5, 1, n)], 1)
