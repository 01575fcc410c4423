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
