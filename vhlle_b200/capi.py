"""ctypes binding of the C ABI in include/vhlle_b200.h (libvhlle_b200.so).

``GpuHydro`` drives one device-resident grid through the C entry points the
way the reference's driver drives Hydro (src/main.cpp:399-428): upload the
initial state, call ``step()`` (== Hydro::performStep) and read fields back.
There is no CPU fallback: constructing a GpuHydro without the built library
or without a GPU raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvhlle_b200.so")

_dp = ctypes.POINTER(ctypes.c_double)

VH_OK, VH_ERR_ARG, VH_ERR_CUDA, VH_ERR_NUMERIC, VH_ERR_STATE = 0, 1, 2, 3, 4

# symbols the header declares (checked by the CPU test suite)
EXPORTS = ("vh_create", "vh_destroy", "vh_set_stream", "vh_upload_state", "vh_download_state",
           "vh_upload_async", "vh_download_async", "vh_device_state", "vh_step", "vh_steps",
           "vh_set_dtau", "vh_get_dtau", "vh_get_tau", "vh_set_tau", "vh_sync",
           "vh_error_bits", "vh_clear_errors", "vh_launches_per_step", "vh_last_error",
           "vh_abi_version", "vh_transform_pv", "vh_eos_eval", "vh_transport_eval", "vh_timer_start", "vh_timer_stop",
           "vh_profile_enable", "vh_profile_read", "vh_profile_kinds", "vh_alloc_pinned",
           "vh_free_pinned", "vh_step_noalloc", "vh_noalloc_last_error", "vh_noalloc_prepare",
           "vh_active_cells", "vh_set_con2prim_method", "vh_init_glauber", "vh_pack_planes",
           "vh_set_surface_eos",
           "vh_unpack_planes",
           "vh_totals",
           "vh_get_grid", "vh_advance", "vh_resize2x", "vh_surface", "vh_surface_begin", "vh_surface_end", "vh_surface_records",
           "vh_surface_device", "vh_surface_write", "vh_enable_vorticity", "vh_vorticity_chain", "vh_get_dbeta",
           "vh_surface_beta", "vh_surface_write_beta", "vh_corona", "vh_cornelius4d", "vh_set_con2prim",
           "vh_con2prim_stats", "vh_mlp_create", "vh_mlp_destroy", "vh_mlp_set_params",
           "vh_mlp_get_params", "vh_mlp_forward", "vh_mlp_grad", "vh_mlp_train",
           "vh_mlp_last_error", "vh_mlp_samples", "vh_set_con2prim_guess", "vh_batch_create",
           "vh_batch_destroy", "vh_batch_set_driver", "vh_batch_tune", "vh_batch_advance",
           "vh_batch_sync", "vh_batch_info", "vh_batch_last_error", "vh_batch_timer_start",
           "vh_batch_timer_stop", "vh_batch_set_mode", "vh_set_slab", "vh_surface_cells",
           "vh_ic_setup_named", "vh_init_glissando", "vh_init_trento", "vh_init_gubser",
           "vh_init_table", "vh_step_host", "vh_init_urqmd")


class VhError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("vhlle_b200 status %d: %s" % (status, msg))
        self.status = status


class VhSurfaceInfo(ctypes.Structure):
    _fields_ = [("nelements", ctypes.c_long), ("nsusp", ctypes.c_long), ("high_T", ctypes.c_long),
                ("EtotSurf", ctypes.c_double), ("nbSurf", ctypes.c_double),
                ("vEff", ctypes.c_double)]


SURF_REC = 29
VH_PLANE_DOUBLES = 47  # doubles per cell moved by vh_pack_planes / vh_unpack_planes


def cornelius4d(cubes, dx, e0, device=0):
    """Device Cornelius on hypercubes [n][16]: (counts[n], cent[n][10][4], norm[n][10][4])."""
    L = lib()
    cubes = np.ascontiguousarray(cubes, dtype=np.float64).reshape(-1, 16)
    n = len(cubes)
    counts = np.zeros(n, dtype=np.int32)
    cent = np.zeros((n, 10, 4))
    norm = np.zeros((n, 10, 4))
    dx = np.ascontiguousarray(dx, dtype=np.float64)
    st = L.vh_cornelius4d(cubes.ctypes.data_as(_dp), n, dx.ctypes.data_as(_dp), e0, device,
                          counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                          cent.ctypes.data_as(_dp), norm.ctypes.data_as(_dp))
    if st != VH_OK:
        raise VhError(st, L.vh_last_error(None).decode())
    return counts, cent, norm


MLP_PARAMS = 4675


def _tensor_ptr(t, dtype_name, shape):
    """Device pointer of a contiguous CUDA tensor of the given dtype and shape."""
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
        raise ValueError("need a contiguous CUDA tensor")
    if str(t.dtype) != "torch." + dtype_name or tuple(t.shape[1:]) != tuple(shape[1:]):
        raise ValueError("need a %s tensor of shape %s" % (dtype_name, shape))
    return ctypes.c_void_p(t.data_ptr())


class Mlp:
    """The learned con2prim start point (vh_mlp_*): 4 -> 64 -> 64 -> 3."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.L = lib()
        h = ctypes.c_void_p()
        st = self.L.vh_mlp_create(device, seed, ctypes.byref(h))
        if st != VH_OK:
            raise VhError(st, self.L.vh_mlp_last_error().decode())
        self.h = h
        self.device = device

    def _check(self, st):
        if st != VH_OK:
            raise VhError(st, self.L.vh_mlp_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.vh_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, dtype=np.float32)
        self._check(self.L.vh_mlp_get_params(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32).reshape(MLP_PARAMS)
        self._check(self.L.vh_mlp_set_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def forward(self, X):
        """X: CUDA float32 [n, 4] -> CUDA float32 [n, 3] (tensor-core path)."""
        import torch
        n = X.shape[0]
        Y = torch.empty((n, 3), dtype=torch.float32, device=X.device)
        self._check(self.L.vh_mlp_forward(self.h, _tensor_ptr(X, "float32", (n, 4)), n,
                                          _tensor_ptr(Y, "float32", (n, 3))))
        return Y

    def grad(self, X, Y):
        n = X.shape[0]
        g = np.zeros(MLP_PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        fp = ctypes.POINTER(ctypes.c_float)
        self._check(self.L.vh_mlp_grad(self.h, _tensor_ptr(X, "float32", (n, 4)),
                                       _tensor_ptr(Y, "float32", (n, 3)), n, g.ctypes.data_as(fp),
                                       ctypes.byref(loss)))
        return g, loss.value

    def train(self, X, Y, batch=16384, epochs=10, lr=3e-3, seed=1):
        n = X.shape[0]
        losses = np.zeros(epochs, dtype=np.float32)
        self._check(self.L.vh_mlp_train(self.h, _tensor_ptr(X, "float32", (n, 4)),
                                        _tensor_ptr(Y, "float32", (n, 3)), n, batch, epochs, lr,
                                        seed, losses.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return losses


class Batch:
    """Independent events advanced together (vh_batch_*): one CUDA graph per
    driver-loop iteration, every event an independent branch."""

    def __init__(self, hydros):
        self.L = lib()
        self.hydros = list(hydros)
        arr = (ctypes.c_void_p * len(self.hydros))(*[h.h.value for h in self.hydros])
        b = ctypes.c_void_p()
        self._check(self.L.vh_batch_create(arr, len(self.hydros), ctypes.byref(b)))
        self.b = b

    def _check(self, st):
        if st != VH_OK:
            raise VhError(st, self.L.vh_batch_last_error().decode())

    def set_driver(self, k, dtau, etamin, etamax, nz, tau_resize=float("inf")):
        self._check(self.L.vh_batch_set_driver(self.b, k, dtau, etamin, etamax, nz, tau_resize))

    def tune(self, enable=True):
        self._check(self.L.vh_batch_tune(self.b, int(enable)))

    def set_mode(self, stage_batched):
        """True: one launch per stage over every event's blocks; False: the
        tuner's configuration (vh_batch_set_mode)."""
        self._check(self.L.vh_batch_set_mode(self.b, int(bool(stage_batched))))

    def advance(self, n=1):
        m = ctypes.c_int()
        for _ in range(n):
            self._check(self.L.vh_batch_advance(self.b, ctypes.byref(m)))
        return m.value

    def sync(self):
        bits = ctypes.c_uint()
        self._check(self.L.vh_batch_sync(self.b, ctypes.byref(bits)))
        return bits.value

    def timer_start(self):
        self._check(self.L.vh_batch_timer_start(self.b))

    def timer_stop(self) -> float:
        ms = ctypes.c_double()
        self._check(self.L.vh_batch_timer_stop(self.b, ctypes.byref(ms)))
        return ms.value

    def info(self):
        c, s, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.L.vh_batch_info(self.b, ctypes.byref(c), ctypes.byref(s), ctypes.byref(b)))
        return {"captures": c.value, "nstreams": s.value, "block": b.value}

    def close(self):
        if getattr(self, "b", None):
            self.L.vh_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VhGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
                ("etamin", ctypes.c_double), ("etamax", ctypes.c_double), ("dz", ctypes.c_double)]


class VhEosAux(ctypes.Structure):
    _fields_ = [("ne", ctypes.c_int), ("nn", ctypes.c_int), ("emin", ctypes.c_double),
                ("emax", ctypes.c_double), ("nmin", ctypes.c_double), ("nmax", ctypes.c_double),
                ("p", _dp), ("T", _dp), ("mub", _dp), ("mus", _dp)]


class VhEosHadron(ctypes.Structure):
    _fields_ = [("ne", ctypes.c_int), ("nnb", ctypes.c_int), ("nnq", ctypes.c_int),
                ("e0", ctypes.c_double), ("n0", ctypes.c_double), ("logemin", ctypes.c_double),
                ("logemax", ctypes.c_double), ("lognmax", ctypes.c_double),
                ("p", _dp), ("T", _dp), ("mub", _dp), ("muq", _dp), ("mus", _dp),
                ("status", ctypes.POINTER(ctypes.c_int))]


class VhEosSmash(ctypes.Structure):
    _fields_ = [("ne", ctypes.c_int), ("nnb", ctypes.c_int), ("nnq", ctypes.c_int),
                ("emin", ctypes.c_double), ("emax", ctypes.c_double), ("nbmin", ctypes.c_double),
                ("nbmax", ctypes.c_double), ("nqmin", ctypes.c_double), ("nqmax", ctypes.c_double),
                ("p", _dp), ("T", _dp), ("mub", _dp), ("muq", _dp), ("mus", _dp)]


class VhEosAzhTable(ctypes.Structure):
    _fields_ = [("ne", ctypes.c_int), ("nn", ctypes.c_int), ("emin", ctypes.c_double),
                ("nmin", ctypes.c_double), ("de", ctypes.c_double), ("dn", ctypes.c_double),
                ("v", _dp)]


class VhEosAzh(ctypes.Structure):
    _fields_ = [(n, VhEosAzhTable) for n in ("p1", "p2", "T1", "T2", "mu1", "mu2")]


class VhEos(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("conf_cnst", ctypes.c_double),
                ("ne", ctypes.c_int), ("nn", ctypes.c_int),
                ("egrid", _dp), ("ngrid", _dp), ("p", _dp), ("T", _dp), ("mub", _dp),
                ("aux", VhEosAux * 2), ("muq", _dp), ("mus", _dp), ("hadron", VhEosHadron),
                ("smash", VhEosSmash), ("azh", VhEosAzh)]


class VhGlauberIc(ctypes.Structure):
    _fields_ = [("parts", _dp), ("nparts", ctypes.c_int), ("smear", ctypes.c_double),
                ("epeak", ctypes.c_double), ("H", _dp), ("ecut", ctypes.c_double),
                ("nb_peak", ctypes.c_double)]


IC_SETUP_FIELDS = ("sNN", "eta0", "sigEta", "etaM", "ybeam", "alphaMix", "Rg", "A", "nsigma",
                   "neta0")


class VhIcSetup(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in IC_SETUP_FIELDS]


class VhGlissandoIc(ctypes.Structure):
    _fields_ = [("setup", VhIcSetup), ("x", _dp), ("y", _dp), ("c", ctypes.POINTER(ctypes.c_int)),
                ("npart", ctypes.POINTER(ctypes.c_int)), ("nevents", ctypes.c_int)]


class VhTrentoIc(ctypes.Structure):
    _fields_ = [("setup", VhIcSetup), ("grid", _dp), ("ngrid", ctypes.POINTER(ctypes.c_int)),
                ("gmax", _dp), ("npart", ctypes.POINTER(ctypes.c_int)), ("nevents", ctypes.c_int)]


class VhTableIc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("x", _dp), ("y", _dp), ("val", _dp),
                ("factor", ctypes.c_double), ("glauber_var", ctypes.c_int)]


class VhUrqmdIc(ctypes.Structure):
    _fields_ = [("p", _dp), ("id", ctypes.POINTER(ctypes.c_int)),
                ("charge", ctypes.POINTER(ctypes.c_int)), ("npart", ctypes.POINTER(ctypes.c_int)),
                ("nevents", ctypes.c_int), ("Rgt", ctypes.c_double), ("Rgz", ctypes.c_double)]


# icModel of the two readers with named setups (src/main.cpp:341-354)
IC_GLISSANDO, IC_TRENTO = 5, 7


def ic_setup(model: int, name: str) -> dict:
    """vh_ic_setup_named: the constants of IcGlissando's (model 5) or
    IcTrento's (model 7) setup `name`, as a dict (ValueError for an unknown
    name, where the reference exits).  Host-only: needs no GPU."""
    out = VhIcSetup()
    if lib().vh_ic_setup_named(model, name.encode(), ctypes.byref(out)) != VH_OK:
        raise ValueError("no setup %r for icModel %d" % (name, model))
    return {n: getattr(out, n) for n in IC_SETUP_FIELDS}


def _ic_setup_struct(d: dict) -> VhIcSetup:
    return VhIcSetup(*[float(d[n]) for n in IC_SETUP_FIELDS])


class VhTrcoeff(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "etaS0", "zetaS0", "ah", "al", "aRho", "T0", "etaSMin", "etaSEpsilonMin",
        "etaSShiftMuB", "etaSScaleMuB", "zetaSPeakEpsilon", "zetaSScaleBeta",
        "zetaSSigmaMinus", "zetaSSigmaPlus")] + [
        ("etaSparam", ctypes.c_int), ("zetaSparam", ctypes.c_int),
        ("zetaSPeakT", ctypes.c_double), ("zetaSWidthT", ctypes.c_double)]


STATE_FIELDS = ("Q", "Qh", "Qprev", "pi", "piH", "Pi", "PiH", "m", "viscCorrCut")
TOTALS = ("E", "Efull", "Nb1", "Nb2", "S", "Px", "vt_num", "vt_den", "vxvy_num", "vxvy_den",
          "pi0x_num", "pi0x_den", "txxyy_num", "txxyy_den", "nCoreCells", "nCoreCutCells")
STATE_NCOMP = dict(Q=7, Qh=7, Qprev=7, pi=10, piH=10, Pi=1, PiH=1, m=3, viscCorrCut=1)


class VhStateView(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in STATE_FIELDS]


_lib = None


def lib():
    """Loads libvhlle_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libvhlle_b200.so is not built (run `python -m vhlle_b200.build`); "
                           "there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.vh_create.argtypes = [ctypes.POINTER(VhGrid), ctypes.POINTER(VhEos),
                            ctypes.POINTER(VhTrcoeff), ctypes.c_double, ctypes.c_double,
                            ctypes.c_int, ctypes.POINTER(vp)]
    L.vh_destroy.argtypes = [vp]
    L.vh_set_stream.argtypes = [vp, vp]
    for n in ("vh_upload_state", "vh_download_state", "vh_upload_async", "vh_download_async",
              "vh_device_state"):
        getattr(L, n).argtypes = [vp, ctypes.POINTER(VhStateView)]
    L.vh_step.argtypes = [vp]
    L.vh_steps.argtypes = [vp, ctypes.c_int]
    L.vh_set_dtau.argtypes = [vp, ctypes.c_double]
    L.vh_get_dtau.argtypes = [vp, _dp]
    L.vh_get_tau.argtypes = [vp, _dp]
    L.vh_set_tau.argtypes = [vp, ctypes.c_double]
    L.vh_sync.argtypes = [vp]
    L.vh_error_bits.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
    L.vh_clear_errors.argtypes = [vp]
    L.vh_launches_per_step.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.vh_last_error.argtypes = [vp]
    L.vh_last_error.restype = ctypes.c_char_p
    L.vh_abi_version.restype = ctypes.c_int
    L.vh_transform_pv.argtypes = [vp, vp, ctypes.c_long, vp]
    L.vh_transport_eval.argtypes = [vp, vp, ctypes.c_long, vp]
    L.vh_timer_start.argtypes = [vp]
    L.vh_timer_stop.argtypes = [vp, _dp]
    L.vh_profile_enable.argtypes = [vp, ctypes.c_int]
    L.vh_profile_read.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                  ctypes.POINTER(ctypes.c_long), _dp]
    L.vh_profile_kinds.restype = ctypes.c_int
    L.vh_alloc_pinned.argtypes = [ctypes.c_size_t, ctypes.POINTER(vp)]
    L.vh_free_pinned.argtypes = [vp]
    L.vh_step_noalloc.argtypes = [ctypes.POINTER(VhGrid), ctypes.POINTER(VhEos),
                                  ctypes.POINTER(VhTrcoeff), ctypes.c_double, ctypes.c_double,
                                  ctypes.POINTER(VhStateView), vp, ctypes.POINTER(ctypes.c_uint)]
    L.vh_noalloc_last_error.restype = ctypes.c_char_p
    L.vh_noalloc_prepare.argtypes = [ctypes.c_int]
    L.vh_active_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.vh_set_con2prim_method.argtypes = [vp, ctypes.c_int]
    L.vh_init_glauber.argtypes = [vp, ctypes.POINTER(VhGlauberIc)]
    L.vh_step_host.argtypes = [vp, ctypes.POINTER(VhStateView), ctypes.POINTER(VhStateView)]
    L.vh_ic_setup_named.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(VhIcSetup)]
    L.vh_init_glissando.argtypes = [vp, ctypes.POINTER(VhGlissandoIc), _dp]
    L.vh_init_trento.argtypes = [vp, ctypes.POINTER(VhTrentoIc), _dp]
    L.vh_init_gubser.argtypes = [vp]
    L.vh_init_table.argtypes = [vp, ctypes.POINTER(VhTableIc)]
    L.vh_init_urqmd.argtypes = [vp, ctypes.POINTER(VhUrqmdIc)]
    L.vh_pack_planes.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
    L.vh_set_surface_eos.argtypes = [vp, ctypes.POINTER(VhEos)]
    L.vh_unpack_planes.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
    L.vh_totals.argtypes = [vp, ctypes.c_double, _dp]
    L.vh_get_grid.argtypes = [vp, ctypes.POINTER(VhGrid)]
    L.vh_advance.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                             ctypes.POINTER(ctypes.c_int)]
    L.vh_resize2x.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.vh_surface.argtypes = [vp, ctypes.c_double, ctypes.POINTER(VhSurfaceInfo)]
    L.vh_corona.argtypes = [vp, ctypes.c_double, ctypes.POINTER(VhSurfaceInfo)]
    L.vh_eos_eval.argtypes = [vp, vp, vp, ctypes.c_long, vp]
    L.vh_surface_begin.argtypes = [vp, ctypes.c_double]
    L.vh_surface_end.argtypes = [vp, ctypes.POINTER(VhSurfaceInfo)]
    L.vh_surface_records.argtypes = [vp, _dp, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
    L.vh_surface_device.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_long)]
    L.vh_surface_write.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    L.vh_enable_vorticity.argtypes = [vp, ctypes.c_int]
    L.vh_get_dbeta.argtypes = [vp, _dp]
    L.vh_vorticity_chain.argtypes = [vp, ctypes.c_int]
    L.vh_surface_beta.argtypes = [vp, _dp, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
    L.vh_surface_write_beta.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    L.vh_set_con2prim.argtypes = [vp, ctypes.c_double]
    L.vh_con2prim_stats.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                    ctypes.POINTER(ctypes.c_ulonglong)]
    fp = ctypes.POINTER(ctypes.c_float)
    L.vh_mlp_create.argtypes = [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(vp)]
    L.vh_mlp_destroy.argtypes = [vp]
    L.vh_mlp_set_params.argtypes = [vp, fp]
    L.vh_mlp_get_params.argtypes = [vp, fp]
    L.vh_mlp_forward.argtypes = [vp, vp, ctypes.c_long, vp]
    L.vh_mlp_grad.argtypes = [vp, vp, vp, ctypes.c_long, fp, fp]
    L.vh_mlp_train.argtypes = [vp, vp, vp, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                               ctypes.c_float, ctypes.c_ulonglong, fp]
    L.vh_mlp_last_error.restype = ctypes.c_char_p
    L.vh_mlp_samples.argtypes = [vp, vp, vp, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
    L.vh_set_con2prim_guess.argtypes = [vp, vp]
    L.vh_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
    L.vh_batch_destroy.argtypes = [vp]
    L.vh_batch_set_driver.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double]
    L.vh_batch_tune.argtypes = [vp, ctypes.c_int]
    L.vh_batch_set_mode.argtypes = [vp, ctypes.c_int]
    L.vh_set_slab.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.vh_surface_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_long,
                                   ctypes.POINTER(ctypes.c_long)]
    L.vh_batch_advance.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.vh_batch_sync.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
    L.vh_batch_info.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 3
    L.vh_batch_last_error.restype = ctypes.c_char_p
    L.vh_batch_timer_start.argtypes = [vp]
    L.vh_batch_timer_stop.argtypes = [vp, _dp]
    L.vh_cornelius4d.argtypes = [_dp, ctypes.c_long, _dp, ctypes.c_double, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int), _dp, _dp]
    _lib = L
    return L


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def make_eos(eos):
    """Lowers a workloads.EosTable into the vh_eos descriptor (arrays kept alive)."""
    d = VhEos()
    d.kind = eos.kind
    d.conf_cnst = eos.conf_cnst
    keep = []
    if eos.kind == 1:
        keep = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (eos.egrid, eos.ngrid, eos.p, eos.T, eos.mub)]
        d.ne, d.nn = len(keep[0]), len(keep[1])
        d.egrid, d.ngrid, d.p, d.T, d.mub = (_ptr(a) for a in keep)
    if eos.kind == 3:
        keep = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (eos.egrid, eos.ngrid, eos.p, eos.T, eos.mub, eos.muq, eos.mus)]
        d.ne, d.nn = len(keep[0]), len(keep[1])
        d.egrid, d.ngrid, d.p, d.T, d.mub, d.muq, d.mus = (_ptr(a) for a in keep)
    if eos.kind == 5:
        keep = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (eos.p, eos.T, eos.mub, eos.muq, eos.mus)]
        h = d.smash
        (h.ne, h.nnb, h.nnq), (eg, bg, qg) = eos.smash
        h.emin, h.emax, h.nbmin, h.nbmax, h.nqmin, h.nqmax = (
            float(eg[0]), float(eg[-1]), float(bg[0]), float(bg[-1]), float(qg[0]), float(qg[-1]))
        h.p, h.T, h.mub, h.muq, h.mus = (_ptr(a) for a in keep)
    if eos.kind == 4:
        keep = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (eos.p, eos.T, eos.mub, eos.muq, eos.mus)]
        st = np.ascontiguousarray(eos.status, dtype=np.int32)
        keep.append(st)
        h = d.hadron
        h.ne, h.nnb, h.nnq, h.e0, h.n0, h.logemin, h.logemax, h.lognmax = eos.hadron
        h.p, h.T, h.mub, h.muq, h.mus = (_ptr(a) for a in keep[:5])
        h.status = st.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    if eos.kind == 6:
        for name, (ne, nn, emin, nmin, de, dn, v) in zip(
                ("p1", "p2", "T1", "T2", "mu1", "mu2"), eos.azh):
            arr = np.ascontiguousarray(v, dtype=np.float64)
            assert arr.size == ne * nn
            keep.append(arr)
            x = getattr(d.azh, name)
            x.ne, x.nn, x.emin, x.nmin, x.de, x.dn = ne, nn, emin, nmin, de, dn
            x.v = _ptr(arr)
    if eos.kind in (2, 7):
        for k, a in enumerate(eos.aux):
            arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (a.p, a.T, a.mub, a.mus)]
            keep += arrs
            x = d.aux[k]
            x.ne, x.nn, x.emin, x.emax, x.nmin, x.nmax = a.ne, a.nn, a.emin, a.emax, a.nmin, a.nmax
            x.p, x.T, x.mub, x.mus = (_ptr(v) for v in arrs)
    return d, keep


def make_trcoeff(setup):
    t = VhTrcoeff()
    for k, v in setup.tr.items():
        setattr(t, k, float(v))
    t.etaSparam = setup.etaSparam
    t.zetaSparam = setup.zetaSparam
    return t


class GpuHydro:
    """One grid on one GPU behind the C ABI (Fluid + Hydro of the reference)."""

    def __init__(self, setup, device: int = 0, upload: bool = True):
        self.L = lib()
        self.setup = setup
        g = setup.grid
        self.N = g.ncells
        grid = VhGrid(g.nx, g.ny, g.nz, *g.bounds(), g.cell_dz or 0.0)
        eos, self._eos_keep = make_eos(setup.eos)
        tr = make_trcoeff(setup)
        h = ctypes.c_void_p()
        st = self.L.vh_create(ctypes.byref(grid), ctypes.byref(eos), ctypes.byref(tr),
                              setup.tau0, setup.dt, device, ctypes.byref(h))
        if st != VH_OK:
            raise VhError(st, self.L.vh_last_error(None).decode())
        self.h = h
        self.device = device
        self._pinned = []
        if upload:
            self.upload_initial()

    def _check(self, st):
        if st != VH_OK:
            raise VhError(st, self.L.vh_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.vh_destroy(self.h)
            self.h = None
        for p in getattr(self, "_pinned", []):
            self.L.vh_free_pinned(p)
        self._pinned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_initial(self):
        """Initial state as the reference ICs leave it: Q, Qprev = Q, all m
        set to the given value, viscous fields zero (src/icGubser.cpp:50-57)."""
        s = self.setup
        Q = np.ascontiguousarray(s.Q, dtype=np.float64).reshape(7, self.N)
        m = np.ascontiguousarray(np.repeat(np.asarray(s.m, dtype=np.float64).reshape(1, self.N), 3, 0))
        fields = dict(Q=Q, m=m)
        if s.pi is not None:
            fields["pi"] = np.ascontiguousarray(s.pi, dtype=np.float64)
        if s.Pi is not None:
            fields["Pi"] = np.ascontiguousarray(s.Pi, dtype=np.float64)
        self.upload(fields)

    def init_glauber(self, parts, H, smear=0.4, epeak=50.0, ecut=1e-3, nb_peak=0.0):
        """vh_init_glauber: the Glauber initial state built on the device from
        the participants' positions parts[n][2] and the longitudinal profile
        H[nz] (workloads.glauber_participants / eta_profile)."""
        parts = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, 2)
        H = np.ascontiguousarray(H, dtype=np.float64).reshape(-1)
        if len(H) != self.setup.grid.nz:
            raise ValueError("H needs one value per eta cell")
        ic = VhGlauberIc(parts.ctypes.data_as(_dp), len(parts), smear, epeak, H.ctypes.data_as(_dp),
                         ecut, nb_peak)
        self._check(self.L.vh_init_glauber(self.h, ctypes.byref(ic)))

    def init_glissando(self, ev, setup: dict):
        """vh_init_glissando: IcGlissando's initial state (icModel 5) from
        ic_files.GlissandoEvents and a setup dict (ic_setup(IC_GLISSANDO,
        name)); returns (sNorm, nNorm)."""
        x = np.ascontiguousarray(ev.x, dtype=np.float64)
        y = np.ascontiguousarray(ev.y, dtype=np.float64)
        c = np.ascontiguousarray(ev.c, dtype=np.int32)
        npart = np.ascontiguousarray(ev.npart, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        ic = VhGlissandoIc(_ic_setup_struct(setup), x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                           c.ctypes.data_as(ip), npart.ctypes.data_as(ip), len(npart))
        norms = np.zeros(2)
        self._check(self.L.vh_init_glissando(self.h, ctypes.byref(ic), norms.ctypes.data_as(_dp)))
        return float(norms[0]), float(norms[1])

    def init_trento(self, ev, setup: dict):
        """vh_init_trento: IcTrento's initial state (icModel 7) from
        ic_files.TrentoEvents and a setup dict; returns (sNorm, nNorm)."""
        grid = np.ascontiguousarray(np.concatenate([np.asarray(g, dtype=np.float64).reshape(-1)
                                                    for g in ev.grids]))
        ngrid = np.array([g.shape[0] for g in ev.grids], dtype=np.int32)
        gmax = np.ascontiguousarray(ev.gmax, dtype=np.float64)
        npart = np.ascontiguousarray(ev.npart, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        ic = VhTrentoIc(_ic_setup_struct(setup), grid.ctypes.data_as(_dp), ngrid.ctypes.data_as(ip),
                        gmax.ctypes.data_as(_dp), npart.ctypes.data_as(ip), len(ngrid))
        norms = np.zeros(2)
        self._check(self.L.vh_init_trento(self.h, ctypes.byref(ic), norms.ctypes.data_as(_dp)))
        return float(norms[0]), float(norms[1])

    def init_gubser(self):
        """vh_init_gubser: ICGubser's initial state (icModel 4)."""
        self._check(self.L.vh_init_gubser(self.h))

    def init_table(self, table, factor=1.0, glauber_var=1):
        """vh_init_table: IC over the s95p table (icModel 2) from an
        ic_files.SongTable."""
        x = np.ascontiguousarray(table.x, dtype=np.float64)
        y = np.ascontiguousarray(table.y, dtype=np.float64)
        val = np.ascontiguousarray(table.val, dtype=np.float64)
        ic = VhTableIc(len(x), len(y), x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                       val.ctypes.data_as(_dp), factor, glauber_var)
        self._check(self.L.vh_init_table(self.h, ctypes.byref(ic)))

    def init_urqmd(self, ev, Rgt=1.0, Rgz=1.0):
        """vh_init_urqmd: IcPartUrqmd's initial state (icModel 3) from
        ic_files.UrqmdEvents with the smearing widths Rgt, Rgz."""
        p = np.ascontiguousarray(ev.p, dtype=np.float64)
        pid = np.ascontiguousarray(ev.id, dtype=np.int32)
        ch = np.ascontiguousarray(ev.charge, dtype=np.int32)
        npart = np.ascontiguousarray(ev.npart, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        ic = VhUrqmdIc(p.ctypes.data_as(_dp), pid.ctypes.data_as(ip), ch.ctypes.data_as(ip),
                       npart.ctypes.data_as(ip), len(npart), Rgt, Rgz)
        self._check(self.L.vh_init_urqmd(self.h, ctypes.byref(ic)))

    def set_surface_eos(self, eos):
        """vh_set_surface_eos: the freeze-out EoS (Fluid's eosH) from a
        workloads.EosTable, or None for the hydro EoS."""
        if eos is None:
            self._check(self.L.vh_set_surface_eos(self.h, None))
            return
        d, keep = make_eos(eos)
        self._check(self.L.vh_set_surface_eos(self.h, ctypes.byref(d)))

    def pack_planes(self, z0, nplanes, buf_ptr):
        """vh_pack_planes into the device buffer at buf_ptr (47 doubles per
        cell of the planes)."""
        self._check(self.L.vh_pack_planes(self.h, z0, nplanes, ctypes.c_void_p(buf_ptr)))

    def unpack_planes(self, z0, nplanes, buf_ptr):
        """vh_unpack_planes from the device buffer at buf_ptr."""
        self._check(self.L.vh_unpack_planes(self.h, z0, nplanes, ctypes.c_void_p(buf_ptr)))

    def set_slab(self, own0, own1, z_global0, nz_global):
        """vh_set_slab: the freeze-out output and the totals of this slab's
        owned planes [own0, own1), its plane 0 being plane z_global0 of a
        grid of nz_global planes."""
        self._check(self.L.vh_set_slab(self.h, own0, own1, z_global0, nz_global))

    def surface_cells(self) -> np.ndarray:
        """[n][3]: the lowest corner (ix, iy, iz of the whole grid) of each
        element's hypercube, for the last vh_surface or vh_corona."""
        n = ctypes.c_long()
        self._check(self.L.vh_surface_cells(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 3), dtype=np.int32)
        if n.value:
            self._check(self.L.vh_surface_cells(
                self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n.value,
                ctypes.byref(n)))
        return out

    def upload(self, fields: dict):
        v = VhStateView()
        keep = []
        for k, a in fields.items():
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(STATE_NCOMP[k], self.N)
            keep.append(a)
            setattr(v, k, a.ctypes.data)
        self._check(self.L.vh_upload_state(self.h, ctypes.byref(v)))

    def step(self, n: int = 1):
        self._check(self.L.vh_steps(self.h, n))

    def sync(self):
        self._check(self.L.vh_sync(self.h))

    def error_bits(self) -> int:
        b = ctypes.c_uint(0)
        self._check(self.L.vh_error_bits(self.h, ctypes.byref(b)))
        return b.value

    @property
    def tau(self) -> float:
        t = ctypes.c_double()
        self._check(self.L.vh_get_tau(self.h, ctypes.byref(t)))
        return t.value

    def set_dtau(self, dt: float):
        self._check(self.L.vh_set_dtau(self.h, dt))

    @property
    def dtau(self) -> float:
        d = ctypes.c_double()
        self._check(self.L.vh_get_dtau(self.h, ctypes.byref(d)))
        return d.value

    def advance(self, dtau: float, etamin: float, etamax: float, nz: int) -> int:
        """The driver's substep block (src/main.cpp:405-419); returns the count."""
        n = ctypes.c_int(0)
        self._check(self.L.vh_advance(self.h, dtau, etamin, etamax, nz, ctypes.byref(n)))
        return n.value

    def resize2x(self) -> int:
        """expandGrid2x (src/main.cpp:246-271): 1 resized, 0 grid not symmetric."""
        r = ctypes.c_int(0)
        self._check(self.L.vh_resize2x(self.h, ctypes.byref(r)))
        return r.value

    def surface(self, ecrit=None):
        """Fluid::outputSurface's freeze-out elements at the current tau:
        (records [n][29], info dict)."""
        info = VhSurfaceInfo()
        ec = self.setup.ecrit if ecrit is None else ecrit
        self._check(self.L.vh_surface(self.h, ec, ctypes.byref(info)))
        return self.surface_records(), {k: getattr(info, k) for k, _ in VhSurfaceInfo._fields_}

    def surface_records(self):
        """The element records [n][29] of the last surface call."""
        n = ctypes.c_long()
        self._check(self.L.vh_surface_records(self.h, None, 0, ctypes.byref(n)))
        rec = np.zeros((n.value, SURF_REC))
        if n.value:
            got = ctypes.c_long()
            self._check(self.L.vh_surface_records(self.h, rec.ctypes.data_as(_dp), n.value,
                                                  ctypes.byref(got)))
        return rec

    def enable_vorticity(self, on=True):
        """Hydro::enableVorticity: dbeta per cell from the next viscous step."""
        self._check(self.L.vh_enable_vorticity(self.h, int(on)))

    def get_dbeta(self):
        """Cell::getDbeta of every cell, [16][N] flattened (4 mu + nu)."""
        out = np.zeros(16 * self.setup.grid.ncells)
        self._check(self.L.vh_get_dbeta(self.h, out.ctypes.data_as(_dp)))
        return out

    def surface_beta(self, ecrit=None):
        """surface() plus the elements' 16 Cartesian d_mu beta_nu of the
        beta.dat lines: (records [n][29], info dict, beta [n][16])."""
        rec, info = self.surface(ecrit)
        n = len(rec)
        beta = np.zeros((n, 16))
        if n:
            got = ctypes.c_long()
            self._check(self.L.vh_surface_beta(self.h, beta.ctypes.data_as(_dp), n,
                                               ctypes.byref(got)))
        return rec, info, beta

    def surface_write_beta(self, path, header=False):
        self._check(self.L.vh_surface_write_beta(self.h, path.encode(), int(header)))

    def set_con2prim_method(self, method):
        """vh_set_con2prim_method: 0 the reference's constant slope, 1 the
        EoS's own slope (tight tolerance only)."""
        self._check(self.L.vh_set_con2prim_method(self.h, int(method)))

    def set_con2prim(self, tol):
        self._check(self.L.vh_set_con2prim(self.h, tol))

    def con2prim_stats(self, enable=True):
        """(calls, iterations) since the last call; keeps counting if enable."""
        c, it = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        self._check(self.L.vh_con2prim_stats(self.h, int(enable), ctypes.byref(c), ctypes.byref(it)))
        return c.value, it.value

    def mlp_samples(self, X, Y):
        """Features and tight labels of every cell into CUDA tensors X [cap, 4],
        Y [cap, 3]; returns the number written."""
        cap = X.shape[0]
        n = ctypes.c_long()
        self._check(self.L.vh_mlp_samples(self.h, _tensor_ptr(X, "float32", (cap, 4)),
                                          _tensor_ptr(Y, "float32", (cap, 3)), cap, ctypes.byref(n)))
        return n.value

    def set_con2prim_guess(self, mlp):
        self._check(self.L.vh_set_con2prim_guess(self.h, mlp.h if mlp is not None else None))

    def transport_eval(self, inp):
        """TransportCoeff::getEta + getTau on the device with this grid's
        transport parameters: inp[n][6] = e, nb, T, muB, s, p -> [n][4] =
        eta/s, zeta/s, tau_pi, tau_Pi (vh_transport_eval)."""
        import torch
        a = np.ascontiguousarray(np.asarray(inp, dtype=np.float64).reshape(-1, 6).T)
        n = a.shape[1]
        dev = "cuda:%d" % self.device
        din = torch.from_numpy(a).to(dev)
        dout = torch.empty((4, n), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self._check(self.L.vh_transport_eval(self.h, ctypes.c_void_p(din.data_ptr()), n,
                                             ctypes.c_void_p(dout.data_ptr())))
        self.sync()
        return dout.cpu().numpy().T.copy()

    def eos6(self, e, nb):
        """The context's EoS on the device (vh_eos_eval): [n][6] = p, T,
        muB, muS, EoS::p, EoS::s (nq = ns = 0)."""
        import torch
        e = np.ascontiguousarray(e, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.float64)
        n = len(e)
        dev = "cuda:%d" % self.device
        de, dn = torch.from_numpy(e).to(dev), torch.from_numpy(nb).to(dev)
        dout = torch.empty((6, n), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self._check(self.L.vh_eos_eval(self.h, ctypes.c_void_p(de.data_ptr()),
                                       ctypes.c_void_p(dn.data_ptr()), n,
                                       ctypes.c_void_p(dout.data_ptr())))
        self.sync()
        return dout.cpu().numpy().T.copy()

    def corona(self, ecrit=None):
        """Fluid::outputCorona's elements at the current tau (vh_corona):
        (records [n][29], info dict)."""
        info = VhSurfaceInfo()
        ec = self.setup.ecrit if ecrit is None else ecrit
        self._check(self.L.vh_corona(self.h, ec, ctypes.byref(info)))
        n = info.nelements
        rec = np.zeros((n, SURF_REC))
        if n:
            got = ctypes.c_long()
            self._check(self.L.vh_surface_records(self.h, rec.ctypes.data_as(_dp), n,
                                                  ctypes.byref(got)))
        return rec, {k: getattr(info, k) for k, _ in VhSurfaceInfo._fields_}

    def surface_only(self, ecrit=None):
        """vh_surface without copying the records: the info dict."""
        info = VhSurfaceInfo()
        ec = self.setup.ecrit if ecrit is None else ecrit
        self._check(self.L.vh_surface(self.h, ec, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in VhSurfaceInfo._fields_}

    def surface_begin(self, ecrit=None):
        """vh_surface_begin: enqueue a surface call; results at surface_end()."""
        ec = self.setup.ecrit if ecrit is None else ecrit
        self._check(self.L.vh_surface_begin(self.h, ec))

    def surface_end(self):
        """vh_surface_end: the info dict of the pending surface call."""
        info = VhSurfaceInfo()
        self._check(self.L.vh_surface_end(self.h, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in VhSurfaceInfo._fields_}

    def surface_write(self, path, extend=False):
        self._check(self.L.vh_surface_write(self.h, path.encode(), int(extend)))

    def grid(self):
        g = VhGrid()
        self._check(self.L.vh_get_grid(self.h, ctypes.byref(g)))
        return g

    def grid_coords(self):
        """getX(0), getX(nx-1), getY(0), getY(ny-1), getZ(0), getZ(nz-1), dx, dy, dz."""
        g = self.grid()
        with np.errstate(all="ignore"):
            a = np.array([g.xmin, g.xmax, g.ymin, g.ymax, g.etamin, g.etamax], dtype=np.float64)
            n = np.array([g.nx - 1, g.ny - 1, g.nz - 1], dtype=np.float64)
            d = (a[1::2] - a[0::2]) / n
            return np.array([a[0] + 0 * d[0], a[0] + n[0] * d[0], a[2] + 0 * d[1],
                             a[2] + n[1] * d[1], a[4] + 0 * d[2], a[4] + n[2] * d[2],
                             d[0], d[1], d[2]])

    def active_cells(self) -> int:
        """Cells the last viscous step relaxed (e > 0 at the half step)."""
        n = ctypes.c_longlong()
        self._check(self.L.vh_active_cells(self.h, ctypes.byref(n)))
        return n.value

    def launches_per_step(self) -> int:
        n = ctypes.c_int()
        self._check(self.L.vh_launches_per_step(self.h, ctypes.byref(n)))
        return n.value

    def step_host(self, fields: dict, sync=True):
        """vh_step_host: one step with the state in the host arrays
        `fields` (name -> float64 array [ncomp][N], uploaded before and
        overwritten after the step); pinned arrays (pinned_state) let the
        copies overlap the kernels."""
        v = VhStateView()
        for k, a in fields.items():
            assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] and a.size == STATE_NCOMP[k] * self.N
            setattr(v, k, a.ctypes.data)
        self._check(self.L.vh_step_host(self.h, ctypes.byref(v), ctypes.byref(v)))
        if sync:
            self.sync()

    def pinned_state(self, fields=STATE_FIELDS) -> dict:
        """Page-locked host arrays (vh_alloc_pinned) for the named fields,
        [ncomp][N] float64; released by close()."""
        out = {}
        for k in fields:
            n = STATE_NCOMP[k] * self.N
            p = ctypes.c_void_p()
            self._check(self.L.vh_alloc_pinned(n * 8, ctypes.byref(p)))
            self._pinned.append(p)
            out[k] = np.ctypeslib.as_array((ctypes.c_double * n).from_address(p.value)).reshape(
                STATE_NCOMP[k], self.N)
        return out

    def get_state(self, fields=STATE_FIELDS) -> dict:
        v = VhStateView()
        out = {}
        for k in fields:
            out[k] = np.empty((STATE_NCOMP[k], self.N))
            setattr(v, k, out[k].ctypes.data)
        self._check(self.L.vh_download_state(self.h, ctypes.byref(v)))
        return out

    def timer_start(self):
        self._check(self.L.vh_timer_start(self.h))

    def timer_stop(self) -> float:
        ms = ctypes.c_double()
        self._check(self.L.vh_timer_stop(self.h, ctypes.byref(ms)))
        return ms.value

    def profile(self, on: bool):
        self._check(self.L.vh_profile_enable(self.h, 1 if on else 0))

    def profile_read(self) -> dict:
        """{kernel name: (launches, total device ms)} since profiling started."""
        out = {}
        for k in range(self.L.vh_profile_kinds()):
            name = ctypes.c_char_p()
            n = ctypes.c_long()
            ms = ctypes.c_double()
            self._check(self.L.vh_profile_read(self.h, k, ctypes.byref(name), ctypes.byref(n),
                                               ctypes.byref(ms)))
            if n.value:
                out[name.value.decode()] = (n.value, ms.value)
        return out

    def totals(self, ecrit=None) -> dict:
        """Interior totals of Fluid::outputSurface for the current state."""
        out = np.zeros(len(TOTALS))
        ec = self.setup.ecrit if ecrit is None else ecrit
        self._check(self.L.vh_totals(self.h, ec, _ptr(out)))
        return dict(zip(TOTALS, out))

    def device_state(self) -> dict:
        v = VhStateView()
        self._check(self.L.vh_device_state(self.h, ctypes.byref(v)))
        return {k: getattr(v, k) for k in STATE_FIELDS}
