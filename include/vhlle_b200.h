/*
 * vhlle_b200.h -- C ABI of the B200 hydro step (libvhlle_b200.so).
 *
 * The library replaces the per-timestep update of the vHLLE hydro code,
 * Hydro::performStep (reference src/hdo.h:55, src/hdo.cpp:1016-1134), and
 * the pieces it calls, with FP64 CUDA kernels for sm_100a that run on a
 * structure-of-arrays grid resident in device memory.  The host keeps the
 * reference's class surface (Hydro / Fluid / EoS / TransportCoeff) and calls
 * down through these entry points; there is no CPU fallback: every entry
 * point that needs the GPU returns VH_ERR_CUDA when there is none.
 *
 * Conventions
 *  - Plain C types, pointers and sizes only.  All functions return a
 *    vh_status; 0 is success.  vh_last_error() gives the message of the last
 *    failure on a context (or of vh_create when ctx is NULL).
 *  - Cell index i = ix + nx*(iy + ny*iz) (x fastest, Fluid::getCell,
 *    src/fld.h:70-78).  Fields are component-major: field[c*N + i].
 *  - pi^{mu nu} is stored as 10 components in index44 order
 *    (src/cll.cpp:22-31): 00,10,11,20,21,22,30,31,32,33.
 *  - Calls on one context are not thread-safe; use one context per thread.
 *  - Device work is enqueued on the context's stream and is asynchronous;
 *    vh_sync() waits and reports numerical failures that the reference
 *    would have stopped on with exit() (NaN fluxes, e > 1e10, ...).
 */
#ifndef VHLLE_B200_H
#define VHLLE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: vh_eos gained the aux tables of VH_EOS_CHIRAL (a caller built against
 * version 1 passes a shorter vh_eos);
 * 3: vh_grid gained dz, vh_eos the EoS3f, EoSHadron, EoSSmash and EoSAZH
 * members (kinds 3-6); kind 7 (EoSCMFe) uses aux */
#define VH_ABI_VERSION 3

typedef int vh_status;
#define VH_OK 0
#define VH_ERR_ARG 1      /* invalid argument (the reference would exit) */
#define VH_ERR_CUDA 2     /* CUDA runtime failure or no usable GPU        */
#define VH_ERR_NUMERIC 3  /* device error word set during a step          */
#define VH_ERR_STATE 4    /* call out of order (e.g. step before upload)  */

/* device error-word bits, returned by vh_error_bits() */
#define VH_NUM_E_HUGE 1u       /* e > 1e10 in hlle_flux, src/hdo.cpp:118-130 */
#define VH_NUM_FLUX_NAN 2u     /* NaN HLLE flux, src/hdo.cpp:285-298        */
#define VH_NUM_SOURCE_NAN 4u   /* NaN source, src/hdo.cpp:345-351           */
#define VH_NUM_NSQUANT_NAN 8u  /* inf/NaN shear, src/hdo.cpp:643-651        */
#define VH_NUM_SURFACE 16u     /* a hypercube on which Cornelius stops the
                                  reference (src/cornelius.cpp:1217,1534) */

typedef struct vh_ctx vh_ctx;

/* Fluid geometry (Fluid ctor arguments, src/fld.h:29-31; dx = (xmax-xmin)/(nx-1)). */
typedef struct vh_grid {
  int nx, ny, nz;
  double xmin, xmax, ymin, ymax, etamin, etamax;
  /* eta cell size: 0 derives it from the bounds as the Fluid constructor
   * does (src/fld.cpp:79); a slab of a larger grid (vh_pack_planes) passes
   * the whole grid's, so that its cells are the whole grid's bit for bit
   * (its bounds then place its planes' coordinates). */
  double dz;
} vh_grid;

/* EoS descriptor.  Device code cannot call the host EoS virtuals
 * (src/eos.h:21-38), so the EoS is lowered to data:
 *  kind VH_EOS_CONFORMAL: p = e/3, T = (e/conf_cnst)^(1/4), muB = 0;
 *  kind VH_EOS_TABLE:     EoS1f (e, nb) table (src/eo1.cpp:21-123): sorted
 *                         egrid[ne], ngrid[nn] (nn >= 2), p/T/mub[ie + ne*inb];
 *  kind VH_EOS_CHIRAL:    EoSChiral (src/eoChiral.cpp:99-178): aux[0] the
 *                         chiralsmall table (used for e < 1.46, nb < 0.3),
 *                         aux[1] the chiraleos table (e < 146, nb < 6), and
 *                         p = 0.2964 e, T = 0.15120476935 e^(1/4) above;
 *  kind VH_EOS_TABLE3:    EoS3f (e, nb, nq, ns) table (src/eo3.cpp:21-175):
 *                         sorted egrid[ne] and ngrid[nn] (one grid for the
 *                         three charges), p/T/mub and muq/mus at
 *                         [ie + ne*ib + ne*nn*iq + ne*nn*nn*is].  The states
 *                         evolved here carry no electric or strange charge
 *                         (no IC sets them and the fluxes keep them zero),
 *                         so the lookups take nq = ns = 0 as the reference's
 *                         transformPV then does;
 *  kind VH_EOS_HADRON:    EoSHadron (src/eoHadron.cpp), the hadronic EoS the
 *                         reference driver gives the freeze-out surface
 *                         (eosTypeHadron 0): `hadron` below;
 *  kind VH_EOS_SMASH:     EoSSmash (src/eoSmash.cpp, eosTypeHadron 1):
 *                         `smash` below; both for vh_set_surface_eos only;
 *  kind VH_EOS_AZH:       EoSAZH (src/eoAZH.cpp, eosType 2): six uniform
 *                         (e, nb) tables, `azh` below;
 *  kind VH_EOS_CMFE:      EoSCMFe (src/eoCMFe.cpp, eosType 4): aux[0] the
 *                         small table (eos/cmfe_small.dat), aux[1] the big
 *                         one (eos/cmfe.dat), converted to GeV/fm^3, fm^-3
 *                         and GeV as its constructor does, in the aux layout
 *                         [in * ne + ie]; a NaN entry is allowed (the
 *                         reference then returns zeros).
 * Host arrays are copied at vh_create (vh_set_surface_eos). */
#define VH_EOS_CONFORMAL 0
#define VH_EOS_TABLE 1
#define VH_EOS_CHIRAL 2
#define VH_EOS_TABLE3 3
#define VH_EOS_HADRON 4
#define VH_EOS_SMASH 5
#define VH_EOS_AZH 6
#define VH_EOS_CMFE 7
/* One EoSaux table (src/eoChiral.cpp:33-97) after its constructor's unit
 * conversions: the e and nb grids are uniform from emin to emax (GeV/fm^3)
 * and nmin to nmax (fm^-3) with ne, nn >= 2 points; p (GeV/fm^3), T, muB,
 * muS (GeV) at [in * ne + ie]. */
typedef struct vh_eos_aux {
  int ne, nn;
  double emin, emax, nmin, nmax;
  const double *p, *T, *mub, *mus;
} vh_eos_aux;
typedef struct vh_eos {
  int kind;
  double conf_cnst;
  int ne, nn;
  const double *egrid, *ngrid, *p, *T, *mub;
  vh_eos_aux aux[2]; /* VH_EOS_CHIRAL and VH_EOS_CMFE only */
  const double *muq, *mus; /* VH_EOS_TABLE3 only */
  /* VH_EOS_HADRON only: the file's header ne nnb nnq e0 n0 logemin logemax
   * lognmax (src/eoHadron.cpp:19) and its tables p, T, muB, muQ, muS and
   * status at [inq + nnq*inb + nnq*nnb*ie] */
  struct vh_eos_hadron {
    int ne, nnb, nnq;
    double e0, n0, logemin, logemax, lognmax;
    const double *p, *T, *mub, *muq, *mus;
    const int *status;
  } hadron;
  /* VH_EOS_SMASH only: ne x nnb x nnq points on uniform grids from emin to
   * emax, nbmin to nbmax, nqmin to nqmax (the first and last rows' values,
   * src/eoSmash.cpp:45-51); p, T, muB, muQ, muS at [inq + nnq*inb +
   * nnq*nnb*ie] */
  struct vh_eos_smash {
    int ne, nnb, nnq;
    double emin, emax, nbmin, nbmax, nqmin, nqmax;
    const double *p, *T, *mub, *muq, *mus;
  } smash;
  /* VH_EOS_AZH only: EoSAZH's six EoSAZHaux tables (src/eoAZH.cpp:15-56),
   * p, T and muB below (1) and above (2) the first table's e range.  Each
   * has ne x nn points on the uniform grids e = emin + ie de, nb = nmin +
   * in dn (ne and nn the file's counts plus one), values at [ie * nn + in]. */
  struct vh_eos_azh {
    struct vh_eos_azh_table {
      int ne, nn;
      double emin, nmin, de, dn;
      const double *v;
    } p1, p2, T1, T2, mu1, mu2;
  } azh;
} vh_eos;

/* TransportCoeff public constants (src/trancoeff.h:8-11, ctor :14-20). */
typedef struct vh_trcoeff {
  double etaS0, zetaS0, ah, al, aRho, T0, etaSMin, etaSEpsilonMin,
      etaSShiftMuB, etaSScaleMuB, zetaSPeakEpsilon, zetaSScaleBeta,
      zetaSSigmaMinus, zetaSSigmaPlus;
  int etaSparam, zetaSparam;
  /* zetaSparam 5 (no counterpart in the reference's src/trancoeff.cpp:32-65):
   * zeta/s = zetaS0 exp(-(T - zetaSPeakT)^2 / (2 zetaSWidthT^2)), a Gaussian
   * bump in T (GeV); unused by the other parameterisations. */
  double zetaSPeakT, zetaSWidthT;
} vh_trcoeff;

/* A view of the per-cell fields (host or device pointers depending on the
 * call).  Any pointer may be NULL to skip that field.  Sizes in doubles:
 * Q, Qh, Qprev 7N; pi, piH 10N; Pi, PiH, viscCorrCut N; m 3N. */
typedef struct vh_state_view {
  double *Q, *Qh, *Qprev, *pi, *piH, *Pi, *PiH, *m, *viscCorrCut;
} vh_state_view;

/* Creates a context on CUDA device `device`, allocates the grid in device
 * memory and uploads the EoS tables.  Replaces the Fluid + Hydro
 * constructors (src/fld.cpp:62-112, src/hdo.cpp:50-57); rejects dt > dx/2 or
 * dt > dy/2 like Hydro::setDtau (src/hdo.cpp:67-75). */
vh_status vh_create(const vh_grid *grid, const vh_eos *eos,
                    const vh_trcoeff *tr, double tau0, double dt, int device,
                    vh_ctx **out);
vh_status vh_destroy(vh_ctx *ctx);

/* The EoS of the freeze-out surface, the corona and the totals: Fluid's
 * eosH, which outputSurface and outputCorona swap in for their whole body
 * (src/fld.cpp:540-542, 870-872, 885-887, 1085-1087); the reference driver
 * passes EoSHadron or EoSSmash there (src/main.cpp:305-311).  eos = NULL
 * goes back to the hydro EoS (the default).  Any kind but the conformal gas;
 * VH_EOS_HADRON and VH_EOS_SMASH only here. */
vh_status vh_set_surface_eos(vh_ctx *ctx, const vh_eos *eos);

/* Uses `stream` (a cudaStream_t, NULL = legacy default) for all later work. */
vh_status vh_set_stream(vh_ctx *ctx, void *stream);

/* Copies cell fields from host memory and synchronises.  Fields left NULL
 * take the values of a freshly initialised cell (src/cll.cpp:33-52) except
 * Qprev, which defaults to Q as after Cell::saveQprev.  Q rows with Q_t < 0
 * are zeroed as by Cell::setQ (src/cll.h:75-80). */
vh_status vh_upload_state(vh_ctx *ctx, const vh_state_view *host);
/* Copies cell fields to host memory and synchronises. */
vh_status vh_download_state(vh_ctx *ctx, const vh_state_view *host);
/* Asynchronous variants on the context stream; host buffers should be
 * pinned (cudaHostAlloc) for the copies to overlap.  No defaults applied:
 * NULL fields are left untouched. */
vh_status vh_upload_async(vh_ctx *ctx, const vh_state_view *host);
vh_status vh_download_async(vh_ctx *ctx, const vh_state_view *host);
/* Device pointers of the resident fields (valid until vh_destroy). */
vh_status vh_device_state(vh_ctx *ctx, vh_state_view *dev);

/* Hydro::performStep (src/hdo.cpp:1016-1134): one timestep of the whole
 * grid; tau advances by dt.  Asynchronous.  The step is captured once
 * (per fill-fraction buffer order, and again after a call that changes
 * what it bakes in) on a private stream and replayed as one CUDA graph
 * launch on the context's stream; with per-kernel profiling on, or if the
 * capture is refused, the kernels are launched one by one. */
vh_status vh_step(vh_ctx *ctx);
/* One performStep with the state in host memory: copies the non-NULL
 * fields of `in` to the device, steps as vh_step, and copies the fields
 * named in `out` back (in and out may be the same view), as one CUDA graph
 * launch on the context's stream whose copies overlap the step's kernels
 * where its data flow allows: Q, m, Qh and Qprev go up first; pi, piH, Pi,
 * PiH and viscCorrCut go up beside the ideal predictor and corrector, which
 * do not read them; m comes back once the step's updateM has run, piH, PiH
 * and viscCorrCut once the relaxation's advection has, the rest at the
 * end.  Asynchronous: the host buffers must stay valid and unread until
 * the work is done (vh_sync), and must be pinned (vh_alloc_pinned) for the
 * copies to overlap anything.  The graph is captured per buffer set (and
 * fill-fraction buffer order) and replayed while they repeat; with
 * profiling on, or if the capture is refused, it is the sequence
 * vh_upload_async, vh_step, vh_download_async.  No defaults are applied to
 * NULL input fields (they keep their device values). */
vh_status vh_step_host(vh_ctx *ctx, const vh_state_view *in, const vh_state_view *out);
/* n successive performStep calls. */
vh_status vh_steps(vh_ctx *ctx, int n);

/* Hydro::setDtau / getDtau / getTau (src/hdo.h:24-26,57). */
vh_status vh_set_dtau(vh_ctx *ctx, double dt);
vh_status vh_get_dtau(vh_ctx *ctx, double *dt);
vh_status vh_get_tau(vh_ctx *ctx, double *tau);
vh_status vh_set_tau(vh_ctx *ctx, double tau);

/* The con2prim (transformPV, src/rmn.cpp:28-139) stopping tolerance on
 * |dv| for every root find of the context: the reference's 1e-5 by default.
 * A tighter value (down to round-off, e.g. 1e-13) makes the result
 * independent of the start point, which is what a learned start point
 * (vh_set_con2prim_guess) needs to stay within 1e-8 of the tight oracle.
 * No counterpart in the reference (its tolerance is a literal). */
vh_status vh_set_con2prim(vh_ctx *ctx, double tol);

/* The con2prim root find's Newton slope.  VH_C2P_REFERENCE (the default):
 * the reference's constant dp/de = 1/3 (src/rmn.cpp:36,96), which converges
 * linearly wherever c_s^2 differs from 1/3.  VH_C2P_TABLE_SLOPE: the EoS's
 * own local derivatives, f'(v) = Q_t + p - v (M dp/de + dp/dnb Q_nb v /
 * sqrt(1 - v^2)), quadratic inside a table cell, with the same bisection
 * safeguard and a stop on an exactly zero residual (the reference's bracket
 * test would send an exact root into bisection).  Only with a tight
 * tolerance (tol <= 1e-10, where the root does not depend on the path to
 * it); it is not the reference's iteration.  Applies to the step's root
 * finds.  No counterpart in the reference. */
#define VH_C2P_REFERENCE 0
#define VH_C2P_TABLE_SLOPE 1
vh_status vh_set_con2prim_method(vh_ctx *ctx, int method);

/* The learned con2prim start point.  A vh_mlp is a 4 -> 64 -> 64 -> 3
 * network (SiLU; BF16 weights and activations, FP32 accumulation) from the
 * features x = (0.1 ln T^00, min(|T^0i|/T^00, 1.5), J^0/T^00,
 * [|T^0i| > T^00]) of T^0mu = Q/tau to (e/T^00, |v|, nb/T^00).  Attached to
 * a context, it runs once per step over every cell (tensor-core tiles) and
 * its |v| becomes the start point of every con2prim root find of that cell
 * in the step; the FP64 safeguarded Newton / bisection still finishes each
 * solve to the context's tolerance, so only the iteration count changes.
 * Use it with a tight tolerance (vh_set_con2prim): at the reference's 1e-5
 * the result depends on the start point.  No counterpart in the reference.
 *
 * Parameters (VH_MLP_PARAMS floats): W1[64][4], b1[64], W2[64][64], b2[64],
 * W3[3][64], b3[3].  vh_mlp_samples writes features X[n][4] and labels
 * Y[n][3] (from the root converged to 1e-13) of every cell of a context
 * with a state into device arrays; vh_mlp_train runs epochs of Adam with a
 * cosine-decayed step on the weighted squared error (weights 1, 4, 1) with
 * the project's own forward / backward kernels and writes each epoch's mean
 * loss to epoch_loss[epochs] (may be NULL); vh_mlp_grad gives the gradient
 * of the mean loss over n samples (for checks); vh_mlp_forward evaluates
 * the inference path.  X, Y are device pointers.  Errors of the vh_mlp_*
 * calls that take no context are described by vh_mlp_last_error(). */
#define VH_MLP_PARAMS 4675
typedef struct vh_mlp vh_mlp;
vh_status vh_mlp_create(int device, unsigned long long seed, vh_mlp **out);
vh_status vh_mlp_destroy(vh_mlp *mlp);
vh_status vh_mlp_set_params(vh_mlp *mlp, const float *params);
vh_status vh_mlp_get_params(vh_mlp *mlp, float *params);
vh_status vh_mlp_forward(vh_mlp *mlp, const float *X, long n, float *Y);
vh_status vh_mlp_grad(vh_mlp *mlp, const float *X, const float *Y, long n,
                      float *grad, float *loss);
vh_status vh_mlp_train(vh_mlp *mlp, const float *X, const float *Y, long n,
                       int batch, int epochs, float lr, unsigned long long seed,
                       float *epoch_loss);
const char *vh_mlp_last_error(void);
vh_status vh_mlp_samples(vh_ctx *ctx, float *X, float *Y, long cap, long *n);
/* Attaches (mlp != NULL) or detaches the start-point network; the context
 * does not own it (destroy it after the context stops using it). */
vh_status vh_set_con2prim_guess(vh_ctx *ctx, vh_mlp *mlp);

/* Counts of con2prim root finds and their iterations since the previous
 * call (read, then reset); enable = 1 keeps counting (slower: two atomics
 * per root find), 0 stops.  For measurements, not production steps. */
vh_status vh_con2prim_stats(vh_ctx *ctx, int enable, unsigned long long *calls,
                            unsigned long long *iters);

/* The grid the context currently evolves: the creation grid, or the one
 * vh_resize2x made, whose bounds are derived from the old grid's first and
 * last cell coordinates exactly as expandGrid2x does. */
vh_status vh_get_grid(vh_ctx *ctx, vh_grid *out);

/* The substep block of the driver loop (src/main.cpp:405-419): while
 * dtau / n > tau * (etamax - etamin) / (nz - 1) the count n doubles; with
 * n > 1 the step is divided by n for n performStep calls and restored, else
 * one performStep runs.  dtau, etamin, etamax and nz are the run
 * parameters (not the resized grid).  *nsub (may be NULL) receives n. */
vh_status vh_advance(vh_ctx *ctx, double dtau, double etamin, double etamax,
                     int nz, int *nsub);

/* expandGrid2x (src/main.cpp:246-271) on the device: same nx, ny, nz over
 * twice the transverse range; every cell imports all variables of the old
 * cell at 2*(i - n/2) + n/2 in x and y (clamped to the grid), and the time
 * step doubles.  A grid whose x or y range is not symmetric is kept
 * (*resized = 0, VH_OK) as the reference does; a doubled step above half
 * the new cell size returns VH_ERR_ARG with nothing changed (the reference
 * exits).  *resized may be NULL. */
vh_status vh_resize2x(vh_ctx *ctx, int *resized);

/* The initial state of a Monte-Carlo Glauber event, built on the device at
 * the context's tau: the participants' density prof(x, y) = sum_p
 * exp(-((x - x_p)^2 + (y - y_p)^2) / (2 smear^2)) on the transverse grid
 * (summed in participant order), normalised to its maximum, e = (epeak
 * H[iz]) prof, cells with e < ecut set to vacuum, nb = (nb_peak H[iz]) prof
 * where e > 0, and every cell set at rest as Cell::setPrimVar + saveQprev +
 * setAllM(e > 0) leave it (src/cll.cpp:222-241, the ending of every IC module
 * such as src/icGlauber.cpp:147-166); the viscous fields start at zero.
 * Replaces the host IC generation plus vh_upload_state.  parts and H are
 * host arrays.  No counterpart in the reference (its Glauber IC is an
 * optical one through GSL). */
typedef struct vh_glauber_ic {
  const double *parts; /* [nparts][2]: x, y of each participant (fm) */
  int nparts;
  double smear;        /* Gaussian width (fm) */
  double epeak;        /* e at the profile's maximum (GeV/fm^3) */
  const double *H;     /* [nz] longitudinal profile of each eta cell */
  double ecut;         /* e below which a cell starts as vacuum */
  double nb_peak;      /* nb at the maximum (fm^-3) */
} vh_glauber_ic;
vh_status vh_init_glauber(vh_ctx *ctx, const vh_glauber_ic *ic);

/* ---- the reference's initial-state modules, built on the device ----
 * Each call replaces the host IC module plus vh_upload_state: it leaves
 * every cell as a fresh Fluid's cell (Cell::Cell, src/cll.cpp:33-52) after
 * the module's setIC, at the context's tau (the driver's tau0).  Per-source
 * and per-cell work (smearing, interpolation, the s95p inversion, the
 * normalisation sums in the reference's loop order, setPrimVar) runs on the
 * device; per-axis factors (nz or nx*nz values of exp, cosh, tanh, sinh)
 * are evaluated once on the host with the C library, as the reference
 * evaluates them.  The modules' console summaries (total energy, angular
 * momentum) are not printed.  A slab context (vh_set_slab) is refused with
 * VH_ERR_STATE: the normalisation sums run over the whole grid. */

/* The collision setup constants of IcGlissando (icModel 5) and IcTrento
 * (icModel 7): src/icGlissando.cpp:33-123, src/icTrento.cpp:33-88.  A setup
 * leaves unset what it does not use (0 here). */
typedef struct vh_ic_setup {
  double sNN;      /* sqrt(s_NN) (GeV): < 100 adds the baryon density, 27
                      recomputes eta0, sigEta, neta0, nsigma per event */
  double eta0;     /* midrapidity plateau */
  double sigEta;   /* diffuseness of the rapidity profile */
  double etaM;     /* tilt of the sources' rapidity profile (IcGlissando) */
  double ybeam;    /* beam rapidity */
  double alphaMix; /* WN / binary mixing */
  double Rg;       /* transverse Gaussian smearing (fm, IcGlissando) */
  double A;        /* initial shear flow (0 in every setup) */
  double nsigma;   /* width of the baryon Gaussian */
  double neta0;    /* centre of the baryon Gaussian */
} vh_ic_setup;
/* The constants of a named setup ("LHC276", "RHIC200", "LHC5020",
 * "RHIC62", "RHIC27", and for IcGlissando "AFTER72") of model 5 or 7;
 * VH_ERR_ARG for another name (where the reference exits). */
vh_status vh_ic_setup_named(int model, const char *name, vh_ic_setup *out);

/* IcGlissando (src/icGlissando.cpp): Gaussian-smeared sources of nevents
 * GLISSANDO events, each spread over +-(int)(3 Rg / dx) cells (cells with
 * ix > 0, iy > 0 only, as the reference's loop) with a tilted, plateau
 * rapidity profile; the entropy normalisation sNorm (and, below 100 GeV,
 * the baryon normalisation nNorm) iterated to a change of at most 1e-4
 * against npart = (all sources) / nevents (integer division); then
 * e = s95p_e(sNorm rho / nevents / dx / dy), nb, nq = 0.4 nb, setPrimVar
 * and setAllM(1) where e > 0; Qprev stays zero.  Host arrays. */
typedef struct vh_glissando_ic {
  vh_ic_setup setup;
  const double *x, *y; /* [nsrc] source positions (fm), every event in file order */
  const int *c;        /* [nsrc] the source's code (non-zero; binary-collision
                          lines, code 0, are dropped by the reader) */
  const int *npart;    /* [nevents] sources of each event (>= 1) */
  int nevents;
} vh_glissando_ic;
/* norms (may be NULL) <- sNorm, nNorm (nNorm 0 above 100 GeV) */
vh_status vh_init_glissando(vh_ctx *ctx, const vh_glissando_ic *ic, double *norms);

/* IcTrento (src/icTrento.cpp): the bilinear interpolation of each TRENTO
 * event's n x n entropy grid over [-grid_max, grid_max]^2 times the plateau
 * rapidity profile, summed over the events; below 2760 GeV sNorm (and below
 * 100 GeV nNorm) iterated against the last event's npart; then
 * e = s95p_e(sNorm rho / nevents) and setPrimVar as IcGlissando.  Host
 * arrays. */
typedef struct vh_trento_ic {
  vh_ic_setup setup;
  const double *grid;   /* every event's n^2 values in file order (row iy, then ix) */
  const int *ngrid;     /* [nevents] n (grid-nsteps, >= 2) */
  const double *gmax;   /* [nevents] grid-max (fm) */
  const int *npart;     /* [nevents] npart of the header */
  int nevents;
} vh_trento_ic;
vh_status vh_init_trento(vh_ctx *ctx, const vh_trento_ic *ic, double *norms);

/* ICGubser (src/icGubser.cpp, icModel 4): the Gubser flow at t = q = 1,
 * e = (4 / (1 + 2 (1 + r^2) + (1 - r^2)^2))^(4/3), transverse velocity
 * 2 r / (2 + r^2) radially, setPrimVar + saveQprev + setAllM. */
vh_status vh_init_gubser(vh_ctx *ctx);

/* IC (src/ic.cpp, icModel 2) over the table of s95p::loadSongIC
 * (src/s95p.cpp:43-88): values val[ix * ny + iy] on the axes x[nx], y[ny]
 * (the first and last entries set the range), times factor and, for
 * glauber_var 1, turned from entropy to energy by s95p_e; bilinear
 * interpolation (zero off the table) times the plateau rapidity factor,
 * cells below e = 0.5 set to vacuum, setPrimVar at rest + saveQprev +
 * setAllM.  Host arrays. */
typedef struct vh_table_ic {
  int nx, ny;
  const double *x, *y, *val;
  double factor;    /* s0ScaleFactor */
  int glauber_var;  /* glauberVar: 1 entropy density, else energy density */
} vh_table_ic;
vh_status vh_init_table(vh_ctx *ctx, const vh_table_ic *ic);

/* IcPartUrqmd (src/icPartUrqmd.cpp, icModel 3): every particle's
 * energy-momentum (mt cosh and sinh of rap - eta + zdiff, px, py), baryon
 * number (+-1 for |id| < 56) and charge smeared over a Gaussian in x, y and
 * eta (widths Rgt, Rgt, Rgz; the eta term dropped for Rgz < 1e-5) on the
 * stencil +-(int)(6 Rgt / dx), +-(int)(6 Rgt / dy), +-(int)(1.5 Rgz / dz)
 * around its rounded cell (cells with ix, iy, iz > 0), normalised to the
 * stencil's own sum, averaged over the events; then per cell transformPV
 * (the reference's Newton at its 1e-5 tolerance), the module's cut (e <
 * 1e-7 or |x| > 10, |y| > 10, |eta| > 5 fm: vacuum), setPrimVar and
 * setAllM; Qprev stays zero.  Host arrays. */
typedef struct vh_urqmd_ic {
  const double *p;     /* [n][8]: tau, x, y, eta, mt, px, py, rap of every event's
                          particles in file order */
  const int *id;       /* [n] particle id */
  const int *charge;   /* [n] */
  const int *npart;    /* [nevents] particles of each event (>= 1) */
  int nevents;
  double Rgt, Rgz;     /* the params keys Rgt and Rgz */
} vh_urqmd_ic;
vh_status vh_init_urqmd(vh_ctx *ctx, const vh_urqmd_ic *ic);

/* One event split into slabs along eta (one context per slab, a GPU each):
 * every persistent field (Q, Qh, Qprev, pi, piH, Pi, PiH, m, viscCorrCut:
 * VH_PLANE_DOUBLES doubles per cell) of the z-planes [z0, z0 + nplanes)
 * into (pack) or out of (unpack) a contiguous DEVICE buffer laid out
 * [field][component][plane][nx * ny], on the context's stream (no wait).
 * A step reaches at most 6 cells along eta (the fill fractions 1, each ideal
 * stage 2, NSquant's neighbours 1, the advection's upwind cell 1, the
 * viscous face flux 1), so slabs that carry 6 halo planes on each inner
 * side and receive them from their neighbours' owned planes once per step
 * evolve their owned planes exactly as the whole grid does.  The slab
 * contexts take the global cell size dz bit for bit (their eta bounds are
 * chosen so).  No counterpart in the reference (it runs on one CPU core). */
#define VH_PLANE_DOUBLES 47
vh_status vh_pack_planes(vh_ctx *ctx, int z0, int nplanes, double *buf_dev);
vh_status vh_unpack_planes(vh_ctx *ctx, int z0, int nplanes, const double *buf_dev);
/* A slab's share of the freeze-out output: its planes [own0, own1) are the
 * ones it owns, and its plane 0 is plane z_global0 of a whole grid of
 * nz_global planes.  vh_surface and vh_corona then take only the
 * hypercubes whose lowest corner is an owned plane (and interior in the
 * whole grid: [2, nz_global - 2)), and vh_totals only the owned interior
 * cells, with Fluid::outputSurface's mid-rapidity window at the whole
 * grid's centre; the slabs' elements are then the whole grid's, and their
 * sums add up to its.  vh_set_slab(ctx, 0, nz, 0, nz) is the whole grid
 * again.  vh_surface_cells gives, for each element of the last vh_surface
 * or vh_corona, the lowest corner (ix, iy, iz of the whole grid) of its
 * hypercube (cap elements at most, *n their number): the slabs' records in
 * order of that cell (iz fastest, a cube's elements in their order) are the
 * whole grid's in its order. */
vh_status vh_set_slab(vh_ctx *ctx, int own0, int own1, int z_global0, int nz_global);
vh_status vh_surface_cells(vh_ctx *ctx, int *ixyz, long cap, long *n);

/* The number of cells the last viscous step relaxed and advected: those
 * with e > 0 at the half step, the cells ISformal does not zero
 * (src/hdo.cpp:694-708); 0 for an ideal context.  Waits for the stream.
 * For measurements (the relaxation's bytes per launch scale with it). */
vh_status vh_active_cells(vh_ctx *ctx, long long *n);

/* Waits for the context's work; returns VH_ERR_NUMERIC if a step set the
 * device error word (then vh_error_bits tells which check fired). */
vh_status vh_sync(vh_ctx *ctx);
vh_status vh_error_bits(vh_ctx *ctx, unsigned *bits);
vh_status vh_clear_errors(vh_ctx *ctx);

/* Number of kernel launches one vh_step issues for this context. */
vh_status vh_launches_per_step(vh_ctx *ctx, int *n);

/* Interior totals that Fluid::outputSurface accumulates and prints after a
 * step (src/fld.cpp:544-604, 846-857), for the current state and tau:
 * out[VH_TOTALS_N] = E, Efull, Nb1, Nb2, S (each already multiplied by
 * dx*dy*dz, as the reference does), Px, vt_num, vt_den, vxvy_num,
 * vxvy_den, pi0x_num, pi0x_den, txxyy_num, txxyy_den, nCoreCells,
 * nCoreCutCells.  e_crit is the freeze-out energy density of the core-cell
 * count.  Waits for the result. */
#define VH_TOTALS_N 16
vh_status vh_totals(vh_ctx *ctx, double ecrit, double *out);

/* The freeze-out hypersurface of Fluid::outputSurface (src/fld.cpp:606-842)
 * at the current tau: every interior cube [ix,ix+1]x[iy,iy+1]x[iz,iz+1]
 * (indices in [2, n-2)) spanning [tau - dt_fluid, tau], with the energy
 * densities of Q at tau and Qprev at tau - dt_fluid at its 16 corners, goes
 * through Cornelius 4D at e_crit; each element gets the 4-linearly
 * interpolated state (con2prim, EoS), its dSigma_mu (built, as in the
 * reference, from the normal of its cube's first element), u^mu, pi^{mu nu}
 * in Cartesian components and Pi.  dt_fluid is the step the grid was
 * created with (doubled by vh_resize2x), not the substep.  Elements are
 * kept on the device in the reference's loop order (ix, iy, iz with iz
 * fastest, then element index) until the next call.  Waits for the result;
 * VH_ERR_NUMERIC if a hypercube would stop the reference (VH_NUM_SURFACE). */
typedef struct vh_surface_info {
  long nelements; /* elements of this call */
  long nsusp;     /* elements with e > 2 e_crit or e < e_crit / 2 */
  long high_T;    /* elements with T > 0.4 or |muB| > 0.85 (the reference
                     prints a warning for each) */
  double EtotSurf; /* energy through the surface, summed over the calls on
                      this grid (a Fluid member: a resize restarts it) */
  double nbSurf;   /* baryon number through the surface, summed over all
                      calls of the context (a function static there) */
  double vEff;     /* effective volume, summed like EtotSurf */
} vh_surface_info;
vh_status vh_surface(vh_ctx *ctx, double ecrit, vh_surface_info *info);

/* The corona of Fluid::outputCorona (src/fld.cpp:876-1089), which the
 * reference driver writes once at tau0, before the first step
 * (src/main.cpp:390): every interior cube whose eight corners have
 * e <= e_crit at the current tau and whose corner-averaged Q / tau gives
 * e >= 0.01 becomes one element at the cube centre with dSigma_mu =
 * tau dx dy deta (cosh eta, 0, 0, -sinh eta) and the corner-averaged state.
 * Its records replace the last vh_surface call's (vh_surface_records,
 * _device and _write return them).  EtotSurf and vEff add to the grid's
 * sums; info->nbSurf is the corona's own running sum (a separate function
 * static in the reference); nsusp is 0; high_T counts T > 0.4 or
 * |muB| > 0.99.  Waits for the result. */
vh_status vh_corona(vh_ctx *ctx, double ecrit, vh_surface_info *info);

/* Element records of the last vh_surface call, VH_SURF_REC doubles each:
 * tau, x, y, eta, dSigma_0..3, u^0..3, T, muB, muQ, muS, pi^{mu nu}
 * (10, index44 order: 00 01 11 02 12 22 03 13 23 33), Pi, e, nb.
 * vh_surface_records copies min(n, max) of them to host memory and sets
 * *n (may be NULL) to n; vh_surface_device gives the device array (valid
 * until the next vh_surface or vh_destroy). */
#define VH_SURF_REC 29
vh_status vh_surface_records(vh_ctx *ctx, double *out, long max, long *n);
vh_status vh_surface_device(vh_ctx *ctx, const double **rec, long *n);
/* vh_surface in two halves, so that a caller can enqueue the next steps
 * before it waits: vh_surface_begin copies the fields the pass reads (Q,
 * Qprev, pi, Pi, and dbeta with vorticity on: 25 or 41 doubles per cell,
 * allocated by the first call) in order on the context stream, then runs
 * the call's kernels and the copy of its counts and sums from that copy on
 * a stream of its own, beside the steps the caller queues next, and
 * returns; vh_surface_end waits for them, orders the context stream after
 * them and fills `info` as vh_surface would (the records stay on the
 * device until the next surface or corona call).  One call in flight per
 * context; vh_surface, vh_corona and the record getters refuse while one is.
 * The call runs with the buffers earlier calls left (64k hypercubes and
 * twice as many elements at first, grown by any call that found more).  If
 * it finds more than they hold, vh_surface_end grows the buffers and runs
 * the pass again on the copy, on the context stream: no call loses
 * elements.
 * While a call is pending, vh_upload_state, vh_upload_async, vh_resize2x,
 * vh_enable_vorticity and vh_set_stream return VH_ERR_STATE. */
vh_status vh_surface_begin(vh_ctx *ctx, double ecrit);
vh_status vh_surface_end(vh_ctx *ctx, vh_surface_info *info);
/* Appends the last call's elements to a text file as freezeout.dat lines
 * (src/fld.cpp:658-797: 15 significant digits, width 24; e and nb only
 * when extendFO). */
vh_status vh_surface_write(vh_ctx *ctx, const char *path, int extendFO);

/* Vorticity.  Replaces Hydro::enableVorticity (src/hdo.cpp:60-64, with
 * Fluid::enableVorticity, src/fld.h:44-52): from the next viscous step on,
 * every step stores d_mu beta_nu (beta = u / T) per cell as ISformal does
 * (src/hdo.cpp:381-611, 682-727), and vh_surface also computes the beta.dat
 * values of its elements.  on = 0 stops the per-step work (the stored
 * values stay).  Cells start at zero, and again after vh_resize2x. */
vh_status vh_enable_vorticity(vh_ctx *ctx, int on);
/* How many earlier lone increments of M[3][0] / M[3][3] (no row-3 write
 * at their cell) one cell follows back before it folds its run by walking
 * the loop positions in order instead (0-32, default 32).  The result is the
 * same either way; for tests of both paths. */
vh_status vh_vorticity_chain(vh_ctx *ctx, int n);
/* Cell::getDbeta of every cell (src/cll.h:199-204): out[(4 mu + nu) * N +
 * i], clamped to [-100, 100] as Cell::setDbeta stores it.  Synchronous. */
vh_status vh_get_dbeta(vh_ctx *ctx, double *out);
/* The last vh_surface call's 16 Cartesian d_i beta_j per element (the
 * beta.dat columns 17-32, src/fld.cpp:798-831), out[min(n, max)][16];
 * *n = the element count.  Synchronous. */
vh_status vh_surface_beta(vh_ctx *ctx, double *out, long max, long *n);
/* Appends the last vh_surface call's elements (none after a vh_corona call)
 * to a text file as beta.dat lines (src/fld.cpp:663-669, 741-745, 826-830:
 * position, dSigma, u, T, muB, muQ, muS, the 16 d_i beta_j, e; 15
 * significant digits, width 24); header != 0
 * first writes Fluid::printDbetaHeader's three lines (src/fld.cpp:174-188),
 * which need a vh_corona call before (its element count is in them). */
vh_status vh_surface_write_beta(vh_ctx *ctx, const char *path, int header);

/* Cornelius::find_surface_4d (src/cornelius.cpp:2247-2285) on n independent
 * hypercubes, on the device: cubes[k][16] corner values (index it*8 + jx*4 +
 * jy*2 + jz, dimension 0 is time), cell sizes dx[4], iso-value e0.
 * counts[k] = element count (-1 where the reference stops), cent and norm
 * [k][10][4] the elements' centroids and normals.  Synchronous; for tests
 * and for callers with their own cubes. */
vh_status vh_cornelius4d(const double *cubes, long n, const double *dx, double e0,
                         int device, int *counts, double *cent, double *norm);

/* Many independent events advanced together (no counterpart in the
 * reference, which runs one event per process).  The batch holds contexts
 * it does not own, all on one device and uploaded; vh_batch_advance runs
 * one iteration of the driver loop for every event -- its substep block
 * (src/main.cpp:405-419, from the event's driver parameters) and, once tau
 * reaches the event's tau_resize, the x2 resize (src/main.cpp:423-427) --
 * as one CUDA graph in which every event is an independent branch.  The
 * graph is captured once per shape (substep counts, buffer parity, launch
 * configuration, context settings) and replayed; results are bit-identical
 * to advancing each context alone with vh_advance / vh_resize2x.
 * vh_batch_set_driver sets an event's (k >= 0) or every event's (k < 0)
 * dtau, eta range, nz and tau_resize (defaults: the context's step and grid,
 * no resize).  A batch has two forms of the iteration: a branch per event
 * over capture streams, or stage-batched: one launch per stage of the step
 * (faces, updates, relaxation, ...) over a work table of every event's
 * blocks, so that hundreds of small grids run as one grid per stage (only
 * when every event has the same EoS class and viscosity and none has
 * vorticity on).  vh_batch_tune(b, 1) times the next iterations under each
 * launch configuration (capture streams and block size of the branch form,
 * and the stage-batched form) and keeps the fastest; vh_batch_set_mode(b,
 * 1) selects the stage-batched form, 0 the tuner's choice (VH_ERR_ARG where
 * the stage-batched form is unavailable); vh_batch_info reports nstreams = 0
 * for it.
 * Set every context (tolerance, network, stream counters) before advancing;
 * a change is picked up by re-capturing.  vh_batch_sync waits and ORs the
 * events' device error words (VH_ERR_NUMERIC if any is set).  Errors of
 * batch calls are described by vh_batch_last_error(). */
typedef struct vh_batch vh_batch;
vh_status vh_batch_create(vh_ctx *const *ctxs, int n, vh_batch **out);
vh_status vh_batch_destroy(vh_batch *batch);
vh_status vh_batch_set_driver(vh_batch *batch, int k, double dtau, double etamin,
                              double etamax, int nz, double tau_resize);
vh_status vh_batch_tune(vh_batch *batch, int enable);
vh_status vh_batch_advance(vh_batch *batch, int *nsub_max);
vh_status vh_batch_sync(vh_batch *batch, unsigned *error_bits);
vh_status vh_batch_info(vh_batch *batch, int *captures, int *nstreams, int *block);
vh_status vh_batch_set_mode(vh_batch *batch, int stage_batched);
/* CUDA-event timing of the batch's stream (stop waits for the stop event). */
vh_status vh_batch_timer_start(vh_batch *batch);
vh_status vh_batch_timer_stop(vh_batch *batch, double *ms);
const char *vh_batch_last_error(void);

/* Device timing with CUDA events recorded on the context's stream.
 * vh_timer_stop waits for the stop event and returns the elapsed time. */
vh_status vh_timer_start(vh_ctx *ctx);
vh_status vh_timer_stop(vh_ctx *ctx, double *ms);

/* Per-kernel timing: while enabled, vh_step records an event after every
 * launch.  vh_profile_read waits for the context's work and returns, for
 * kernel kind `kind` (0 <= kind < vh_profile_kinds()), its name, the number
 * of launches and their summed device time since profiling was enabled. */
vh_status vh_profile_enable(vh_ctx *ctx, int on);
vh_status vh_profile_read(vh_ctx *ctx, int kind, const char **name,
                          long *launches, double *total_ms);
int vh_profile_kinds(void);

/* Page-locked host memory for the asynchronous copies. */
vh_status vh_alloc_pinned(size_t bytes, void **p);
vh_status vh_free_pinned(void *p);

const char *vh_last_error(vh_ctx *ctx);
int vh_abi_version(void);

/* Batched con2prim + EoS on device arrays (transformPV, src/rmn.cpp:28-139):
 * Q[7][n] (component-major) -> prim[8][n] = e, p, nb, nq, ns, vx, vy, vz.
 * Uses the context's EoS and stream. */
vh_status vh_transform_pv(vh_ctx *ctx, const double *Q_dev, long n,
                          double *prim_dev);

/* The context's EoS on device arrays (EoS::eos with muS, EoS::p and
 * EoS::s with nq = ns = 0; src/eos.h:21-38, src/eos.cpp:18-25):
 * e[n], nb[n] -> out[6][n] = p, T, muB, muS, p(), s.  Uses the context's
 * stream. */
vh_status vh_eos_eval(vh_ctx *ctx, const double *e_dev, const double *nb_dev, long n,
                      double *out_dev);

/* Batched transport coefficients on device arrays (TransportCoeff::getEta
 * and getTau, src/trancoeff.cpp:68-100) with the context's parameters:
 * in[6][n] = e, nb, T, muB, s, p -> out[4][n] = eta/s, zeta/s, tau_pi,
 * tau_Pi.  Uses the context's stream. */
vh_status vh_transport_eval(vh_ctx *ctx, const double *in_dev, long n,
                            double *out_dev);

/* Allocation-free step.  No counterpart in the reference: this entry point
 * exists for callers that cannot let a library allocate -- host codes whose
 * device memory is reserved up front by their own pool or by another
 * framework's caching allocator, or that forbid cudaMalloc once their time
 * loop runs.  It performs one Hydro::performStep on caller-owned DEVICE
 * arrays: every field of `state` is required (sizes as in vh_state_view),
 * and the EoS table pointers in `eos_dev` are device pointers.  `tau` is the
 * time at the start of the step; the caller advances it by dt.
 * All scratch lives in one static device array sized for at most
 * VH_NOALLOC_MAX_CELLS cells and VH_NOALLOC_MAX_DIM cells per dimension
 * (about 21 MB held on every GPU that loads the library until exit); larger
 * grids are rejected with VH_ERR_ARG.  Nothing is allocated: no cudaMalloc,
 * cudaFree, host malloc or library allocator is called.  The array is a
 * module variable: the CUDA runtime maps it (and loads the step kernels)
 * when the library's module is first used on a device, which with lazy
 * module loading (the default) is the first look-up of its address.  Call
 * vh_noalloc_prepare(device) once per device before reserving your own
 * device memory pool and before any stream capture: it does that look-up
 * and the kernels' set-up, so that later calls take no device memory at
 * all.  Without it, the first vh_step_noalloc call on a device does the
 * same set-up (and may then fail for lack of memory).  Every call on a
 * device shares the array: calls whose GPU work overlaps race, so serialise
 * them.  The call waits for `stream`, writes the device error word to
 * *error_bits (if not NULL) and returns VH_ERR_NUMERIC when it is nonzero;
 * vh_noalloc_last_error() describes the last failure on this thread. */
#define VH_NOALLOC_MAX_CELLS 32768
#define VH_NOALLOC_MAX_DIM 1024
vh_status vh_step_noalloc(const vh_grid *grid, const vh_eos *eos_dev,
                          const vh_trcoeff *tr, double tau, double dt,
                          const vh_state_view *state, void *stream,
                          unsigned *error_bits);
const char *vh_noalloc_last_error(void);
/* The set-up of vh_step_noalloc on CUDA device `device` (made current for
 * the call and restored after): maps the scratch array, looks up its
 * address and sets the step kernels' attributes.  Idempotent. */
vh_status vh_noalloc_prepare(int device);

#ifdef __cplusplus
}
#endif
#endif /* VHLLE_B200_H */
