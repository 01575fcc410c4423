"""ctypes bindings to the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Two checkers are exposed with the same driving interface:

  * ``OracleRun``  the C restatement (oracle/liboracle.so, vh_oracle.c)
  * ``RefRun``     the reference's own hot-path sources compiled unmodified
                   into oracle/_ref/libvhlle_ref.so (present only where the
                   reference tree was available at build time)
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvhlle_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class _Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
                ("zmin", ctypes.c_double), ("zmax", ctypes.c_double), ("dz", ctypes.c_double)]


class _Aux(ctypes.Structure):
    _fields_ = [("ne", ctypes.c_int), ("nn", ctypes.c_int), ("emin", ctypes.c_double),
                ("emax", ctypes.c_double), ("nmin", ctypes.c_double), ("nmax", ctypes.c_double),
                ("p", _dp), ("T", _dp), ("mub", _dp), ("mus", _dp)]


class _Azh(ctypes.Structure):
    _fields_ = [("ne", ctypes.c_int), ("nn", ctypes.c_int), ("emin", ctypes.c_double),
                ("nmin", ctypes.c_double), ("de", ctypes.c_double), ("dn", ctypes.c_double),
                ("v", _dp)]


class _Eos(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("conf_cnst", ctypes.c_double),
                ("ne", ctypes.c_int), ("nn", ctypes.c_int),
                ("egrid", _dp), ("ngrid", _dp), ("p", _dp), ("T", _dp), ("mub", _dp),
                ("tol", ctypes.c_double), ("aux", _Aux * 2), ("crmath", ctypes.c_int),
                ("muq", _dp), ("mus", _dp),
                ("hne", ctypes.c_int), ("hnnb", ctypes.c_int), ("hnnq", ctypes.c_int),
                ("he0", ctypes.c_double), ("hn0", ctypes.c_double), ("logemin", ctypes.c_double),
                ("logemax", ctypes.c_double), ("lognmax", ctypes.c_double),
                ("status", ctypes.POINTER(ctypes.c_int)),
                ("semin", ctypes.c_double), ("semax", ctypes.c_double), ("snbmin", ctypes.c_double),
                ("snbmax", ctypes.c_double), ("snqmin", ctypes.c_double), ("snqmax", ctypes.c_double),
                ("az", _Azh * 6)]


class _Trc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "etaS0", "zetaS0", "ah", "al", "aRho", "T0", "etaSMin", "etaSEpsilonMin",
        "etaSShiftMuB", "etaSScaleMuB", "zetaSPeakEpsilon", "zetaSScaleBeta",
        "zetaSSigmaMinus", "zetaSSigmaPlus")] + [
        ("etaSparam", ctypes.c_int), ("zetaSparam", ctypes.c_int),
        ("zetaSPeakT", ctypes.c_double), ("zetaSWidthT", ctypes.c_double),
        ("crmath", ctypes.c_int)]


class _State(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("Q", "Qh", "Qprev", "pi", "piH", "Pi", "PiH", "m", "vcc",
                                   "dbeta")]


class _IcSetup(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("sNN", "eta0", "sigEta", "etaM", "ybeam",
                                                "alphaMix", "Rg", "A", "nsigma", "neta0")]


_ip = ctypes.POINTER(ctypes.c_int)
_lib_oracle = None
_lib_ref = None


def oracle_lib():
    global _lib_oracle
    if _lib_oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: run `make -C oracle liboracle.so`")
        lib = ctypes.CDLL(ORACLE_SO)
        lib.or_step.restype = ctypes.c_int
        lib.or_step.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.POINTER(_Trc),
                                ctypes.POINTER(_State), _dp, ctypes.c_double]
        lib.or_transform_pv.argtypes = [ctypes.POINTER(_Eos), _dp, ctypes.c_int, _dp]
        lib.or_transport_eval.argtypes = [ctypes.POINTER(_Trc), _dp, ctypes.c_int, _dp]
        lib.or_eos_eval.argtypes = [ctypes.POINTER(_Eos), _dp, _dp, ctypes.c_int, _dp]
        lib.or_eos6.argtypes = [ctypes.POINTER(_Eos), _dp, _dp, ctypes.c_int, _dp]
        lib.or_eos_full.argtypes = [ctypes.POINTER(_Eos), _dp, ctypes.c_int, _dp]
        lib.or_eos_s.argtypes = [ctypes.POINTER(_Eos), _dp, _dp, ctypes.c_int, _dp]
        lib.or_update_m.argtypes = [ctypes.POINTER(_Grid), _dp, ctypes.c_double, ctypes.c_double]
        lib.or_resize2x.restype = ctypes.c_int
        lib.or_resize2x.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_State),
                                    ctypes.POINTER(_Grid), ctypes.POINTER(_State)]
        lib.or_surface.restype = ctypes.c_long
        lib.or_surface.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.POINTER(_State),
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_long,
                                   _dp]
        lib.or_surface_beta.restype = ctypes.c_long
        lib.or_surface_beta.argtypes = lib.or_surface.argtypes + [_dp]
        lib.or_corona.restype = ctypes.c_long
        lib.or_corona.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.POINTER(_State),
                                  ctypes.c_double, ctypes.c_double, _dp, ctypes.c_long, _dp]
        lib.or_cornelius4d.restype = ctypes.c_int
        lib.or_cornelius4d.argtypes = [_dp, _dp, ctypes.c_double, _dp, _dp]
        lib.or_substeps.restype = ctypes.c_int
        lib.or_substeps.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int]
        lib.or_totals.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.POINTER(_Trc),
                                  ctypes.POINTER(_State), ctypes.c_double, ctypes.c_double, _dp]
        lib.or_pow_cr.restype = ctypes.c_double
        lib.or_pow_cr.argtypes = [ctypes.c_double, ctypes.c_double]
        lib.or_s95p_e.restype = ctypes.c_double
        lib.or_s95p_e.argtypes = [ctypes.c_double, ctypes.c_int]
        lib.or_ic_glissando.restype = ctypes.c_int
        lib.or_ic_glissando.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos),
                                        ctypes.POINTER(_IcSetup), ctypes.c_double, _dp, _dp, _ip,
                                        _ip, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_State), _dp]
        lib.or_ic_trento.restype = ctypes.c_int
        lib.or_ic_trento.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos),
                                     ctypes.POINTER(_IcSetup), ctypes.c_double, _dp, _ip, _dp, _ip,
                                     ctypes.c_int, ctypes.c_int, ctypes.POINTER(_State), _dp]
        lib.or_ic_gubser.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.c_double,
                                     ctypes.c_int, ctypes.POINTER(_State)]
        lib.or_ic_urqmd.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.c_double,
                                    _dp, _ip, _ip, _ip, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.POINTER(_State)]
        lib.or_ic_table.argtypes = [ctypes.POINTER(_Grid), ctypes.POINTER(_Eos), ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, ctypes.POINTER(_State)]
        _lib_oracle = lib
    return _lib_oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _lib_ref
    if _lib_ref is None:
        if not ref_available():
            raise RuntimeError("compiled reference not present (oracle/_ref)")
        lib = ctypes.CDLL(REF_SO)
        lib.ref_create.restype = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_char_p, _dp, ctypes.c_int, ctypes.c_int]
        lib.ref_destroy.argtypes = [ctypes.c_void_p]
        lib.ref_set_state.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.ref_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ref_tau.restype = ctypes.c_double
        lib.ref_tau.argtypes = [ctypes.c_void_p]
        lib.ref_set_dtau.restype = ctypes.c_int
        lib.ref_set_dtau.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ref_get_state.argtypes = [ctypes.c_void_p] + [_dp] * 9
        lib.ref_transform_pv.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, _dp]
        lib.ref_transport_eval.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, _dp]
        lib.ref_set_prim_var.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, _dp]
        lib.ref_eos_full.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, _dp]
        lib.ref_surface_eos_full.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, _dp]
        lib.ref_set_surface_eos.restype = ctypes.c_int
        lib.ref_set_surface_eos.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.ref_output_corona.restype = ctypes.c_int
        lib.ref_output_corona.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                          ctypes.c_char_p, ctypes.c_int]
        lib.ref_eos.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int, _dp, _dp]
        lib.ref_eos6.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int, _dp]
        lib.ref_update_m.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        lib.ref_ic.restype = ctypes.c_int
        lib.ref_ic.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p,
                               ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                               _dp, _dp, _dp]
        lib.ref_s95p_e.argtypes = [_dp, ctypes.c_int, _dp]
        lib.ref_totals.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp]
        lib.ref_cornelius4d.restype = ctypes.c_int
        lib.ref_cornelius4d.argtypes = [_dp, _dp, ctypes.c_double, _dp, _dp]
        lib.ref_enable_vorticity.argtypes = [ctypes.c_void_p]
        lib.ref_get_dbeta.argtypes = [ctypes.c_void_p, _dp]
        lib.ref_print_dbeta_header.restype = ctypes.c_int
        lib.ref_print_dbeta_header.argtypes = [ctypes.c_void_p]
        lib.ref_resize2x.restype = ctypes.c_int
        lib.ref_resize2x.argtypes = [ctypes.c_void_p]
        lib.ref_advance.restype = ctypes.c_int
        lib.ref_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int]
        lib.ref_dtau.restype = ctypes.c_double
        lib.ref_dtau.argtypes = [ctypes.c_void_p]
        lib.ref_grid.argtypes = [ctypes.c_void_p, _dp]
        lib.ref_output_surface.restype = ctypes.c_int
        lib.ref_output_surface.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                           ctypes.c_int]
        _lib_ref = lib
    return _lib_ref


FIELDS = ("Q", "Qh", "Qprev", "pi", "piH", "Pi", "PiH", "m", "vcc")
# one freeze-out element record (Fluid::outputSurface, src/fld.cpp:656-797)
SURF_REC = 29
SURF_COLS = ("tau", "x", "y", "eta", "ds0", "ds1", "ds2", "ds3", "u0", "u1", "u2", "u3", "T",
             "mub", "muq", "mus", "pi00", "pi01", "pi11", "pi02", "pi12", "pi22", "pi03", "pi13",
             "pi23", "pi33", "Pi", "e", "nb")
SURF_ACC = ("nsusp", "EtotSurf", "nbSurf", "vEff", "highT")


def cornelius4d(cube, dx, e0, reference=False):
    """One hypercube through the oracle's Cornelius (or the reference's):
    (centroids [n][4], normals [n][4]); n = -1 where the reference stops."""
    cube = np.ascontiguousarray(cube, dtype=np.float64).reshape(16)
    dx = np.ascontiguousarray(dx, dtype=np.float64)
    cent = np.zeros((10, 4))
    norm = np.zeros((10, 4))
    if reference:
        n = ref_lib().ref_cornelius4d(_ptr(cube), _ptr(dx), e0, _ptr(cent), _ptr(norm))
    else:
        n = oracle_lib().or_cornelius4d(_ptr(cube), _ptr(dx), e0, _ptr(cent), _ptr(norm))
    return (cent[:n].copy(), norm[:n].copy()) if n >= 0 else (None, None)


def read_freezeout(path, extend=False):
    """Element records of a freezeout.dat written by the reference
    (src/fld.cpp:658-797: 15 significant digits, OUTPI layout)."""
    rows = []
    with open(path) as f:
        for line in f:
            v = line.split()
            if v:
                rows.append([float(x) for x in v])
    a = np.array(rows, dtype=np.float64).reshape(-1, 29 if extend else 27)
    return a
TOTALS = ("E", "Efull", "Nb1", "Nb2", "S", "Px", "vt_num", "vt_den", "vxvy_num", "vxvy_den",
          "pi0x_num", "pi0x_den", "txxyy_num", "txxyy_den", "nCoreCells", "nCoreCutCells")
FIELD_NCOMP = dict(Q=7, Qh=7, Qprev=7, pi=10, piH=10, Pi=1, PiH=1, m=3, vcc=1)


def empty_state(N):
    return {k: np.zeros((FIELD_NCOMP[k], N)) for k in FIELDS}


def initial_state(setup):
    """Cell contents right after the initial condition: Q, Qprev = Q,
    m = setAllM(value), pi = Pi = 0, viscCorrCut = 1 (src/cll.cpp:33-52)."""
    N = setup.grid.ncells
    st = empty_state(N)
    Q = np.array(setup.Q, dtype=np.float64).reshape(7, N)
    # Cell::setQ zeroing (src/cll.h:75-86)
    neg = Q[0] < 0
    Q[:, neg] = 0.0
    st["Q"][:] = Q
    st["Qprev"][:] = Q
    st["m"][:] = np.asarray(setup.m, dtype=np.float64).reshape(1, N)
    if setup.pi is not None:
        st["pi"][:] = setup.pi
    if setup.Pi is not None:
        st["Pi"][0] = setup.Pi
    st["vcc"][:] = 1.0
    return st


class _EosHolder:
    def __init__(self, eos):
        self.keep = []
        self.s = _Eos()
        self.s.kind = eos.kind
        self.s.conf_cnst = eos.conf_cnst
        if eos.kind == 1:
            arrs = [np.ascontiguousarray(a, dtype=np.float64)
                    for a in (eos.egrid, eos.ngrid, eos.p, eos.T, eos.mub)]
            self.keep = arrs
            self.s.ne = len(arrs[0])
            self.s.nn = len(arrs[1])
            self.s.egrid, self.s.ngrid, self.s.p, self.s.T, self.s.mub = (_ptr(a) for a in arrs)
        if eos.kind == 3:
            arrs = [np.ascontiguousarray(a, dtype=np.float64)
                    for a in (eos.egrid, eos.ngrid, eos.p, eos.T, eos.mub, eos.muq, eos.mus)]
            self.keep = arrs
            self.s.ne = len(arrs[0])
            self.s.nn = len(arrs[1])
            (self.s.egrid, self.s.ngrid, self.s.p, self.s.T, self.s.mub, self.s.muq,
             self.s.mus) = (_ptr(a) for a in arrs)
        if eos.kind == 5:
            arrs = [np.ascontiguousarray(a, dtype=np.float64)
                    for a in (eos.p, eos.T, eos.mub, eos.muq, eos.mus)]
            self.keep = arrs
            (self.s.hne, self.s.hnnb, self.s.hnnq), (eg, bg, qg) = eos.smash
            self.s.semin, self.s.semax = float(eg[0]), float(eg[-1])
            self.s.snbmin, self.s.snbmax = float(bg[0]), float(bg[-1])
            self.s.snqmin, self.s.snqmax = float(qg[0]), float(qg[-1])
            self.s.p, self.s.T, self.s.mub, self.s.muq, self.s.mus = (_ptr(a) for a in arrs)
        if eos.kind == 4:
            arrs = [np.ascontiguousarray(a, dtype=np.float64)
                    for a in (eos.p, eos.T, eos.mub, eos.muq, eos.mus)]
            st = np.ascontiguousarray(eos.status, dtype=np.int32)
            self.keep = arrs + [st]
            (self.s.hne, self.s.hnnb, self.s.hnnq, self.s.he0, self.s.hn0, self.s.logemin,
             self.s.logemax, self.s.lognmax) = eos.hadron
            self.s.p, self.s.T, self.s.mub, self.s.muq, self.s.mus = (_ptr(a) for a in arrs)
            self.s.status = st.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        if eos.kind == 6:
            for k, (ne, nn, emin, nmin, de, dn, v) in enumerate(eos.azh):
                arr = np.ascontiguousarray(v, dtype=np.float64)
                assert arr.size == ne * nn
                self.keep.append(arr)
                x = self.s.az[k]
                x.ne, x.nn, x.emin, x.nmin, x.de, x.dn = ne, nn, emin, nmin, de, dn
                x.v = _ptr(arr)
        if eos.kind in (2, 7):
            for k, a in enumerate(eos.aux):
                arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (a.p, a.T, a.mub, a.mus)]
                self.keep += arrs
                x = self.s.aux[k]
                x.ne, x.nn, x.emin, x.emax, x.nmin, x.nmax = a.ne, a.nn, a.emin, a.emax, a.nmin, a.nmax
                x.p, x.T, x.mub, x.mus = (_ptr(v) for v in arrs)


def _trc(setup, crmath=False):
    t = _Trc()
    for k, v in setup.tr.items():
        setattr(t, k, float(v))
    t.etaSparam = setup.etaSparam
    t.zetaSparam = setup.zetaSparam
    t.crmath = int(crmath)
    return t


def oracle_ic(setup, model, data=None, ic_setup=None, crmath=False, factor=1.0, glauber_var=1,
              Rgt=1.0, Rgz=1.0):
    """The C restatement of an IC module (vh_oracle_ic.c) on setup's grid and
    EoS at setup.tau0: model 5 IcGlissando (data: ic_files.GlissandoEvents),
    7 IcTrento (ic_files.TrentoEvents), 4 ICGubser, 2 IC over a table
    (ic_files.SongTable, factor, glauber_var), 3 IcPartUrqmd
    (ic_files.UrqmdEvents, Rgt, Rgz).  ic_setup: the setup dict of
    models 5 and 7.  Returns (state dict, (sNorm, nNorm))."""
    lib = oracle_lib()
    g = setup.grid
    grid = _Grid(g.nx, g.ny, g.nz, *g.bounds(), g.cell_dz or 0.0)
    eos = _EosHolder(setup.eos)
    eos.s.crmath = int(crmath)
    st = empty_state(g.ncells)
    sv = _State()
    for k in FIELDS:
        setattr(sv, k, _ptr(st[k]))
    norms = np.zeros(2)
    if model in (5, 7):
        su = _IcSetup(*[float(ic_setup[n]) for n, _ in _IcSetup._fields_])
    if model == 5:
        x = np.ascontiguousarray(data.x, dtype=np.float64)
        y = np.ascontiguousarray(data.y, dtype=np.float64)
        c = np.ascontiguousarray(data.c, dtype=np.int32)
        npart = np.ascontiguousarray(data.npart, dtype=np.int32)
        rc = lib.or_ic_glissando(ctypes.byref(grid), ctypes.byref(eos.s), ctypes.byref(su),
                                 setup.tau0, _ptr(x), _ptr(y), c.ctypes.data_as(_ip),
                                 npart.ctypes.data_as(_ip), len(npart), int(crmath),
                                 ctypes.byref(sv), _ptr(norms))
        assert rc == 0
    elif model == 7:
        src = np.ascontiguousarray(np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1)
                                                   for a in data.grids]))
        ngrid = np.array([a.shape[0] for a in data.grids], dtype=np.int32)
        gmax = np.ascontiguousarray(data.gmax, dtype=np.float64)
        npart = np.ascontiguousarray(data.npart, dtype=np.int32)
        rc = lib.or_ic_trento(ctypes.byref(grid), ctypes.byref(eos.s), ctypes.byref(su),
                              setup.tau0, _ptr(src), ngrid.ctypes.data_as(_ip), _ptr(gmax),
                              npart.ctypes.data_as(_ip), len(ngrid), int(crmath), ctypes.byref(sv),
                              _ptr(norms))
        assert rc == 0
    elif model == 3:
        pp = np.ascontiguousarray(data.p, dtype=np.float64)
        pid = np.ascontiguousarray(data.id, dtype=np.int32)
        ch = np.ascontiguousarray(data.charge, dtype=np.int32)
        npart = np.ascontiguousarray(data.npart, dtype=np.int32)
        lib.or_ic_urqmd(ctypes.byref(grid), ctypes.byref(eos.s), setup.tau0, _ptr(pp),
                        pid.ctypes.data_as(_ip), ch.ctypes.data_as(_ip), npart.ctypes.data_as(_ip),
                        len(npart), float(Rgt), float(Rgz), int(crmath), ctypes.byref(sv))
    elif model == 4:
        lib.or_ic_gubser(ctypes.byref(grid), ctypes.byref(eos.s), setup.tau0, int(crmath),
                         ctypes.byref(sv))
    elif model == 2:
        x = np.ascontiguousarray(data.x, dtype=np.float64)
        y = np.ascontiguousarray(data.y, dtype=np.float64)
        val = np.ascontiguousarray(data.val, dtype=np.float64)
        lib.or_ic_table(ctypes.byref(grid), ctypes.byref(eos.s), setup.tau0, len(x), len(y),
                        _ptr(x), _ptr(y), _ptr(val), float(factor), int(glauber_var), int(crmath),
                        ctypes.byref(sv))
    else:
        raise ValueError("no IC model %d" % model)
    return st, (float(norms[0]), float(norms[1]))


class OracleRun:
    """The C restatement driven like Hydro: step() == performStep()."""

    def __init__(self, setup, tol=None, vorticity=False, crmath=False, surface_eos=None):
        """tol: the transformPV stopping tolerance (None: the reference's
        1e-5; a smaller value gives the tight-tolerance oracle).  vorticity:
        Hydro::enableVorticity, d_mu beta_nu per cell in self.dbeta.
        crmath: exp and x^(1/4) in the transport coefficients and EoSChiral's
        power law correctly rounded, as the CUDA path evaluates them (False:
        the C library's, as the reference does)."""
        self.setup = setup
        g = setup.grid
        self.grid = _Grid(g.nx, g.ny, g.nz, *g.bounds(), g.cell_dz or 0.0)
        self.eos = _EosHolder(setup.eos)
        self.eos.s.tol = 0.0 if tol is None else float(tol)
        self.eos.s.crmath = int(crmath)
        # Fluid's eosH: the EoS of the surface, corona and totals (SWAP_EOS,
        # src/fld.cpp:540-542); the hydro EoS unless given
        self.eosH = self.eos
        if surface_eos is not None:
            self.eosH = _EosHolder(surface_eos)
            self.eosH.s.tol = self.eos.s.tol
            self.eosH.s.crmath = int(crmath)
        self.trc = _trc(setup, crmath)
        self.state = initial_state(setup)
        self.tau = ctypes.c_double(setup.tau0)
        self.dt = setup.dt
        self.lib = oracle_lib()
        self.errors = 0
        self.dbeta = np.zeros(16 * g.ncells) if vorticity else None

    def _sview(self):
        s = _State()
        for k in FIELDS:
            setattr(s, k, _ptr(self.state[k]))
        if self.dbeta is not None:
            s.dbeta = _ptr(self.dbeta)
        return s

    def step(self, n=1):
        sv = self._sview()
        for _ in range(n):
            self.errors |= self.lib.or_step(ctypes.byref(self.grid), ctypes.byref(self.eos.s),
                                            ctypes.byref(self.trc), ctypes.byref(sv),
                                            ctypes.byref(self.tau), self.dt)
        return self.errors

    @property
    def tau_now(self):
        return self.tau.value

    def set_dtau(self, dt):
        """Hydro::setDtau (src/hdo.cpp:67-75); returns False instead of exiting."""
        g = self.grid
        dx = (g.xmax - g.xmin) / (g.nx - 1)
        dy = (g.ymax - g.ymin) / (g.ny - 1)
        if dt > dx / 2. or dt > dy / 2.:
            return False
        self.dt = dt
        return True

    def advance(self, dtau, etamin, etamax, nz):
        """The driver's substep block (src/main.cpp:405-419); returns the count."""
        n = self.lib.or_substeps(dtau, self.tau.value, etamin, etamax, nz)
        if n < 0:
            raise RuntimeError("substep count overflow")
        if n > 1:
            self.dt = self.dt / n
            self.step(n)
            self.dt = self.dt * n
        else:
            self.step(1)
        return n

    def resize2x(self):
        """expandGrid2x (src/main.cpp:246-271): 1 resized, 0 not symmetric,
        -1 the doubled step fails the dx/2 check."""
        out = {k: np.empty_like(v) for k, v in self.state.items()}
        so = _State()
        for k in FIELDS:
            setattr(so, k, _ptr(out[k]))
        gout = _Grid()
        si = self._sview()
        if not self.lib.or_resize2x(ctypes.byref(self.grid), ctypes.byref(si), ctypes.byref(gout),
                                    ctypes.byref(so)):
            return 0
        dt2 = 2.0 * self.dt
        dx = (gout.xmax - gout.xmin) / (gout.nx - 1)
        dy = (gout.ymax - gout.ymin) / (gout.ny - 1)
        if dt2 > dx / 2. or dt2 > dy / 2.:
            return -1
        self.grid = gout
        self.state = out
        self.dt = dt2
        if self.dbeta is not None:  # the new fluid's cells start at zero
            self.dbeta = np.zeros_like(self.dbeta)
        return 1

    def grid_coords(self):
        """getX(0), getX(nx-1), getY(0), getY(ny-1), getZ(0), getZ(nz-1), dx, dy, dz."""
        g = self.grid
        with np.errstate(all="ignore"):
            a = np.array([g.xmin, g.xmax, g.ymin, g.ymax, g.zmin, g.zmax], dtype=np.float64)
            n = np.array([g.nx - 1, g.ny - 1, g.nz - 1], dtype=np.float64)
            d = (a[1::2] - a[0::2]) / n
            out = np.array([a[0] + 0 * d[0], a[0] + n[0] * d[0], a[2] + 0 * d[1], a[2] + n[1] * d[1],
                            a[4] + 0 * d[2], a[4] + n[2] * d[2], d[0], d[1], d[2]])
        return out

    def get_state(self):
        return {k: v.copy() for k, v in self.state.items()}

    def totals(self):
        out = np.zeros(len(TOTALS))
        sv = self._sview()
        self.lib.or_totals(ctypes.byref(self.grid), ctypes.byref(self.eosH.s), ctypes.byref(self.trc),
                           ctypes.byref(sv), self.tau.value, self.setup.ecrit, _ptr(out))
        return dict(zip(TOTALS, out))

    def surface(self, dtf=None, cap=200000):
        """Freeze-out elements of outputSurface at the current tau: (records
        [n][29], acc dict).  dtf is the Fluid's step (default: the setup's)."""
        dtf = self.setup.dt if dtf is None else dtf
        rec = np.zeros((cap, SURF_REC))
        acc = np.zeros(5)
        sv = self._sview()
        n = self.lib.or_surface(ctypes.byref(self.grid), ctypes.byref(self.eosH.s), ctypes.byref(sv),
                                self.tau.value, dtf, self.setup.ecrit, _ptr(rec), cap, _ptr(acc))
        if n < 0:
            raise RuntimeError("Cornelius stopped (the reference would exit)")
        assert n <= cap
        return rec[:n].copy(), dict(zip(SURF_ACC, acc))

    def surface_beta(self, dtf=None, cap=200000):
        """surface() plus each element's 16 Cartesian d_mu beta_nu of the
        beta.dat line: (records, acc dict, beta [n][16])."""
        if self.dbeta is None:
            raise RuntimeError("vorticity is off")
        dtf = self.setup.dt if dtf is None else dtf
        rec = np.zeros((cap, SURF_REC))
        beta = np.zeros((cap, 16))
        acc = np.zeros(5)
        sv = self._sview()
        n = self.lib.or_surface_beta(ctypes.byref(self.grid), ctypes.byref(self.eosH.s),
                                     ctypes.byref(sv), self.tau.value, dtf, self.setup.ecrit,
                                     _ptr(rec), cap, _ptr(acc), _ptr(beta))
        if n < 0:
            raise RuntimeError("Cornelius stopped (the reference would exit)")
        assert n <= cap
        return rec[:n].copy(), dict(zip(SURF_ACC, acc)), beta[:n].copy()

    def corona(self, cap=2000000):
        """Fluid::outputCorona's elements at the current tau: (records
        [n][29], acc dict)."""
        rec = np.zeros((cap, SURF_REC))
        acc = np.zeros(5)
        sv = self._sview()
        n = self.lib.or_corona(ctypes.byref(self.grid), ctypes.byref(self.eosH.s), ctypes.byref(sv),
                               self.tau.value, self.setup.ecrit, _ptr(rec), cap, _ptr(acc))
        assert n <= cap
        return rec[:n].copy(), dict(zip(SURF_ACC, acc))

    def transform_pv(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float64).reshape(-1, 7)
        out = np.zeros((len(Q), 8))
        self.lib.or_transform_pv(ctypes.byref(self.eos.s), _ptr(Q), len(Q), _ptr(out))
        return out

    def transport_eval(self, inp):
        """TransportCoeff::getEta + getTau: inp[n][6] = e, nb, T, muB, s, p
        -> [n][4] = eta/s, zeta/s, tau_pi, tau_Pi."""
        inp = np.ascontiguousarray(inp, dtype=np.float64).reshape(-1, 6)
        out = np.zeros((len(inp), 4))
        self.lib.or_transport_eval(ctypes.byref(self.trc), _ptr(inp), len(inp), _ptr(out))
        return out

    def eos_full(self, pts):
        """EoS::eos at pts[n][4] = e, nb, nq, ns -> [n][5] = p, T, muB, muQ, muS."""
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 4)
        out = np.zeros((len(pts), 5))
        self.lib.or_eos_full(ctypes.byref(self.eos.s), _ptr(pts), len(pts), _ptr(out))
        return out

    def eos6(self, e, nb):
        """[n][6] = p, T, muB, muS, EoS::p, EoS::s (nq = ns = 0)."""
        return _eos6(self.lib.or_eos6, ctypes.byref(self.eos.s), e, nb)

    def eos_eval(self, e, nb):
        e = np.ascontiguousarray(e, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.float64)
        out = np.zeros((len(e), 3))
        s = np.zeros(len(e))
        self.lib.or_eos_eval(ctypes.byref(self.eos.s), _ptr(e), _ptr(nb), len(e), _ptr(out))
        self.lib.or_eos_s(ctypes.byref(self.eos.s), _ptr(e), _ptr(nb), len(e), _ptr(s))
        return out, s


def _eos6(fn, h, e, nb):
    e = np.ascontiguousarray(e, dtype=np.float64)
    nb = np.ascontiguousarray(nb, dtype=np.float64)
    out = np.zeros((len(e), 6))
    fn(h, _ptr(e), _ptr(nb), len(e), _ptr(out))
    return out


class RefRun:
    """The compiled reference (Fluid/Hydro objects) behind the same interface."""

    def __init__(self, setup, eos_file=None, surface_eos=None):
        self.setup = setup
        self.h = None
        self._tmp = None
        # TransportCoeff::zetaS (src/trancoeff.cpp:19-70) has branches for
        # zetaSparam 0..4 only and returns no value for any other; the
        # Gaussian bump (5) exists in the oracle alone
        if not 0 <= setup.zetaSparam <= 4 or not 0 <= setup.etaSparam <= 3:
            raise ValueError("the reference has no etaSparam %d / zetaSparam %d"
                             % (setup.etaSparam, setup.zetaSparam))
        self.lib = ref_lib()
        g = setup.grid
        self._tmp = None
        if setup.eos.kind == 1 and eos_file is None:
            self._tmp = tempfile.TemporaryDirectory()
            eos_file = os.path.join(self._tmp.name, "eos1f.dat")
            setup.eos.write_eos1f(eos_file)
        if setup.eos.kind == 3 and eos_file is None:
            self._tmp = tempfile.TemporaryDirectory()
            eos_file = os.path.join(self._tmp.name, "eos3f.dat")
            setup.eos.write_eos3f(eos_file)
        if setup.eos.kind == 2 and eos_file is None:  # the directory that holds eos/
            self._tmp = tempfile.TemporaryDirectory()
            eos_file = self._tmp.name
            setup.eos.write_chiral(eos_file)
        if setup.eos.kind == 6 and eos_file is None:  # the directory that holds eos/
            self._tmp = tempfile.TemporaryDirectory()
            eos_file = self._tmp.name
            setup.eos.write_azh(eos_file)
        if setup.eos.kind == 7 and eos_file is None:  # the directory that holds eos/
            self._tmp = tempfile.TemporaryDirectory()
            eos_file = self._tmp.name
            setup.eos.write_cmfe(eos_file)
        bounds = np.array(g.bounds(), dtype=np.float64)
        tr = np.array(setup.tr_vector(), dtype=np.float64)
        self.h = self.lib.ref_create(g.nx, g.ny, g.nz, _ptr(bounds), setup.tau0, setup.dt,
                                     setup.ecrit, setup.eos.kind, setup.eos.conf_cnst,
                                     (eos_file or "").encode(), _ptr(tr), setup.etaSparam,
                                     setup.zetaSparam)
        if surface_eos is not None:  # Fluid's eosH (kind 4: EoSHadron)
            if self._tmp is None:
                self._tmp = tempfile.TemporaryDirectory()
            hfile = os.path.join(self._tmp.name, "eos_hadron.dat")
            dims = (0, 0, 0)
            if surface_eos.kind == 5:
                surface_eos.write_smash(hfile)
                dims = surface_eos.smash[0]
            else:
                surface_eos.write_hadron(hfile)
            if self.lib.ref_set_surface_eos(self.h, surface_eos.kind, hfile.encode(), *dims) != 0:
                raise ValueError("the reference has no surface EoS of kind %d" % surface_eos.kind)
        st = initial_state(setup)
        self.lib.ref_set_state(self.h, _ptr(st["Q"]), _ptr(st["pi"]), _ptr(st["piH"]),
                               _ptr(st["Pi"][0]), _ptr(st["PiH"][0]), _ptr(st["m"][0].copy()))

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        self.lib.ref_step(self.h, n)
        return 0

    def ic(self, model, path="", setup_name="", s0scale=1.0, glauber_var=1, Rgt=1.0, Rgz=1.0):
        """The reference's IC module `model` (2, 3, 4, 5 or 7:
        src/main.cpp:324-366) on a fresh Fluid of this run's grid, from the
        file at path with the named setup (or the smearing widths Rgt, Rgz);
        returns Q, Qprev [7][N] and m [N] of every cell."""
        N = self.setup.grid.ncells
        Q, Qp, m = np.zeros((7, N)), np.zeros((7, N)), np.zeros(N)
        rc = self.lib.ref_ic(self.h, model, path.encode(), setup_name.encode(), s0scale,
                             glauber_var, Rgt, Rgz, _ptr(Q), _ptr(Qp), _ptr(m))
        if rc != 0:
            raise ValueError("the reference has no IC model %d here" % model)
        return {"Q": Q, "Qprev": Qp, "m": m}

    def s95p_e(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        out = np.zeros_like(s)
        self.lib.ref_s95p_e(_ptr(s), len(s), _ptr(out))
        return out

    def enable_vorticity(self):
        """Hydro::enableVorticity; before the first output_surface call."""
        self.lib.ref_enable_vorticity(self.h)

    def get_dbeta(self):
        """Cell::getDbeta of every cell, [16][N] flattened (4 mu + nu)."""
        out = np.zeros(16 * self.setup.grid.ncells)
        self.lib.ref_get_dbeta(self.h, _ptr(out))
        return out

    def print_dbeta_header(self):
        """Fluid::printDbetaHeader into beta.dat; False when it throws."""
        return self.lib.ref_print_dbeta_header(self.h) == 0

    @property
    def tau_now(self):
        return self.lib.ref_tau(self.h)

    @property
    def dtau(self):
        return self.lib.ref_dtau(self.h)

    def advance(self, dtau, etamin, etamax, nz):
        return self.lib.ref_advance(self.h, dtau, etamin, etamax, nz)

    def resize2x(self):
        return self.lib.ref_resize2x(self.h)

    def grid_coords(self):
        out = np.zeros(9)
        self.lib.ref_grid(self.h, _ptr(out))
        return out

    def get_state(self):
        N = self.setup.grid.ncells
        st = empty_state(N)
        self.lib.ref_get_state(self.h, *[_ptr(st[k]) for k in FIELDS])
        return st

    def transform_pv(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float64).reshape(-1, 7)
        out = np.zeros((len(Q), 8))
        self.lib.ref_transform_pv(self.h, _ptr(Q), len(Q), _ptr(out))
        return out

    def set_prim_var(self, inp):
        """Cell::setPrimVar on n points: inp[n][8] = tau, e, nb, nq, ns, vx,
        vy, vz -> the stored Q [n][7]."""
        inp = np.ascontiguousarray(inp, dtype=np.float64).reshape(-1, 8)
        out = np.zeros((len(inp), 7))
        self.lib.ref_set_prim_var(self.h, _ptr(inp), len(inp), _ptr(out))
        return out

    def transport_eval(self, inp):
        inp = np.ascontiguousarray(inp, dtype=np.float64).reshape(-1, 6)
        out = np.zeros((len(inp), 4))
        self.lib.ref_transport_eval(self.h, _ptr(inp), len(inp), _ptr(out))
        return out

    def totals(self):
        out = np.zeros(len(TOTALS))
        self.lib.ref_totals(self.h, self.tau_now, _ptr(out))
        return dict(zip(TOTALS, out))

    def output_surface(self, outdir, extend=False):
        """Fluid::outputSurface: returns (nelements, printed totals line).
        Element lines go to outdir/freezeout.dat.unfinished."""
        buf = ctypes.create_string_buffer(512)
        n = self.lib.ref_output_surface(self.h, outdir.encode(), int(extend), buf, 512)
        return n, buf.value.decode()

    def output_corona(self, outdir, extend=False):
        """Fluid::outputCorona: returns (nelements, printed totals line).
        Element lines go to outdir/freezeout.dat.unfinished."""
        buf = ctypes.create_string_buffer(512)
        n = self.lib.ref_output_corona(self.h, outdir.encode(), int(extend), buf, 512)
        return n, buf.value.decode()

    def eos6(self, e, nb):
        """[n][6] = p, T, muB, muS, EoS::p, EoS::s (nq = ns = 0)."""
        return _eos6(self.lib.ref_eos6, self.h, e, nb)

    def eos_full(self, pts):
        """EoS::eos at pts[n][4] = e, nb, nq, ns -> [n][5] = p, T, muB, muQ, muS."""
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 4)
        out = np.zeros((len(pts), 5))
        self.lib.ref_eos_full(self.h, _ptr(pts), len(pts), _ptr(out))
        return out

    def surface_eos_full(self, pts):
        """eos_full of the surface EoS (Fluid's eosH)."""
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 4)
        out = np.zeros((len(pts), 5))
        self.lib.ref_surface_eos_full(self.h, _ptr(pts), len(pts), _ptr(out))
        return out

    def eos_eval(self, e, nb):
        e = np.ascontiguousarray(e, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.float64)
        out = np.zeros((len(e), 3))
        s = np.zeros(len(e))
        self.lib.ref_eos(self.h, _ptr(e), _ptr(nb), len(e), _ptr(out), _ptr(s))
        return out, s
