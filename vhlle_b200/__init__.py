"""vhlle_b200: B200-native FP64 kernels for the per-timestep update of the
vHLLE relativistic viscous hydro code (Hydro::performStep), behind a C ABI
(include/vhlle_b200.h) and a thin host layer that keeps the reference's
Hydro / Fluid / EoS / TransportCoeff surface."""

__all__ = ["workloads", "capi"]
