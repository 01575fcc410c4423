"""The C ABI library: builds, loads, exports every entry point that
include/vhlle_b200.h declares, validates arguments before touching a GPU,
and refuses to run without one (no CPU fallback).  No device compute here."""
import ctypes
import os
import re

import pytest

from vhlle_b200 import build as B
from vhlle_b200 import capi
from vhlle_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return capi.lib()


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "vhlle_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vh_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_binding_list():
    assert declared_symbols() == sorted(capi.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.vh_abi_version() == 3


def _create(setup, dt=None):
    L = capi.lib()
    g = setup.grid
    grid = capi.VhGrid(g.nx, g.ny, g.nz, *g.bounds())
    eos, keep = capi.make_eos(setup.eos)
    tr = capi.make_trcoeff(setup)
    h = ctypes.c_void_p()
    st = L.vh_create(ctypes.byref(grid), ctypes.byref(eos), ctypes.byref(tr), setup.tau0,
                     setup.dt if dt is None else dt, 0, ctypes.byref(h))
    msg = L.vh_last_error(None).decode()
    if st == capi.VH_OK:
        L.vh_destroy(h)
    return st, msg


def test_rejects_too_big_timestep_like_setDtau(lib):
    s = W.gubser_setup(nx=21, ny=21)  # dx = 0.5
    st, msg = _create(s, dt=0.3)
    assert st == capi.VH_ERR_ARG and "delta_tau" in msg


def test_rejects_single_column_eos_table(lib):
    s = W.small_glauber3d(9, 5)
    s.eos = W.EosTable(kind=1, egrid=s.eos.egrid, ngrid=s.eos.ngrid[:1], p=s.eos.p[:len(s.eos.egrid)],
                       T=s.eos.T[:len(s.eos.egrid)], mub=s.eos.mub[:len(s.eos.egrid)])
    st, msg = _create(s)
    assert st == capi.VH_ERR_ARG and "nn >= 2" in msg


def test_no_gpu_means_error_not_fallback(lib):
    st, msg = _create(W.gubser_setup(nx=21, ny=21))
    if st == capi.VH_OK:
        pytest.skip("a GPU is present")
    assert st == capi.VH_ERR_CUDA, msg
    with pytest.raises(capi.VhError):
        capi.GpuHydro(W.gubser_setup(nx=21, ny=21))


def test_null_arguments_are_errors(lib):
    L = capi.lib()
    assert L.vh_step(None) == capi.VH_ERR_ARG
    assert L.vh_sync(None) == capi.VH_ERR_ARG
    assert L.vh_destroy(None) == capi.VH_OK
