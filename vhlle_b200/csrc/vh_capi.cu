// vh_capi.cu -- the C ABI declared in include/vhlle_b200.h.
//
// A context owns one fluid grid resident in device memory (the role of the
// reference's Fluid + Hydro pair, src/fld.cpp:62-112, src/hdo.cpp:50-57):
// every field is a component-major FP64 array, the EoS table is copied to
// the device once, and vh_step enqueues the kernels of one performStep on
// the context's stream.  Errors are returned as status codes; nothing in
// here exits or traps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "../../include/vhlle_b200.h"
#include "vh_mlp.cuh"
#include "vh_step.cuh"
#include "vh_surface.cuh"

namespace vh {
void launch_fill(double* p, long long n, double v, cudaStream_t s);
void launch_zero_negative_rows(double* Q, long long N, cudaStream_t s);
}  // namespace vh

#include "vh_ctx.cuh"

namespace {
struct EventMarker : vh::LaunchMarker {
  vh_ctx* c;
  size_t prev;
  cudaError_t err = cudaSuccess;
  EventMarker(vh_ctx* ctx, size_t start) : c(ctx), prev(start) {}
  void after(int kind) override {
    if (c->evused == c->evpool.size()) {
      cudaEvent_t e;
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) {
        err = r;
        return;
      }
      c->evpool.push_back(e);
    }
    const size_t k = c->evused++;
    cudaError_t r = cudaEventRecord(c->evpool[k], c->stream);
    if (r != cudaSuccess) err = r;
    c->segs.push_back({kind, prev, k});
    prev = k;
  }
};
}  // namespace

static thread_local std::string g_create_error;

static vh_status fail(vh_ctx* c, vh_status st, const std::string& msg) {
  if (c)
    c->err = msg;
  else
    g_create_error = msg;
  return st;
}

// Calls that change the grid, its fields' meaning or the stream are refused
// while a vh_surface_begin has not ended: its pass reads the grid and may
// run again at vh_surface_end (the reference takes the surface of the old
// Fluid before a resize replaces it, src/main.cpp:246-271,420-427).
#define VH_NOT_PENDING(ctx, who)                                                   \
  do {                                                                             \
    if ((ctx)->surf_pending)                                                       \
      return fail((ctx), VH_ERR_STATE, who ": a vh_surface_begin has not ended"); \
  } while (0)

static vh_status cuda_fail(vh_ctx* c, cudaError_t e, const char* where) {
  return fail(c, VH_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define VH_CUDA(c, call)                                 \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

template <typename T>
static vh_status dalloc(vh_ctx* c, T** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc");
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return VH_OK;
}

// Replaces *p by an allocation of at least `need` elements (no copy).
template <typename T>
static vh_status dgrow(vh_ctx* c, T** p, size_t* cap, size_t need) {
  if (*p && *cap >= need) return VH_OK;
  if (*p) {
    for (auto it = c->allocs.begin(); it != c->allocs.end(); ++it)
      if (*it == (void*)*p) {
        c->allocs.erase(it);
        break;
      }
    cudaFree(*p);
    *p = nullptr;
  }
  const size_t n = std::max<size_t>(need, 2 * *cap);
  vh_status st = dalloc(c, p, n);
  if (st == VH_OK) *cap = n;
  return st;
}

// Per-dimension source map of the ghost-cell copies: the reference copies
// cell 2 into 1 and 0, then cell n-3 into n-2 and n-1, each index clamped
// into [0, n-1] (src/fld.cpp:211-273).  Simulating that sequence gives, for
// every index, the original cell its final value comes from.
static void ghost_map(int n, int* src, unsigned char* dst) {
  for (int i = 0; i < n; i++) {
    src[i] = i;
    dst[i] = 0;
  }
  auto cl = [n](int i) { return std::min(std::max(i, 0), n - 1); };
  int s = cl(2);
  for (int d : {cl(1), cl(0)}) {
    src[d] = src[s];
    dst[d] = 1;
  }
  s = cl(n - 3);
  for (int d : {cl(n - 2), cl(n - 1)}) {
    src[d] = src[s];
    dst[d] = 1;
  }
}

// Chooses how the device searches a table axis: the index guess of a log
// or linear fit when every grid point is predicted within two places (and
// the axis is strictly increasing), else the reference's binary search.
// Results are identical in every mode; only the number of loads differs.
static void choose_axis_mode(const double* g, int n, int* mode, float* x0, float* inv) {
  *mode = vh::GRID_BSEARCH;
  *x0 = 0.f;
  *inv = 0.f;
  if (n < 3) return;
  for (int k = 1; k < n; k++)
    if (!(g[k] > g[k - 1])) return;
  auto worst = [&](int m, float a0, float ainv) {
    float w = 0.f;
    for (int k = 0; k < n; k++) {
      const float fx = (float)g[k];
      const float t = (m == vh::GRID_LOG ? std::log2(fx) - a0 : fx - a0) * ainv;
      w = std::max(w, std::fabs(t - (float)k));
    }
    return w;
  };
  if (g[0] > 0.) {
    const float a0 = std::log2((float)g[0]);
    const float ainv = (float)(n - 1) / (std::log2((float)g[n - 1]) - a0);
    if (std::isfinite(ainv) && worst(vh::GRID_LOG, a0, ainv) <= 2.f) {
      *mode = vh::GRID_LOG;
      *x0 = a0;
      *inv = ainv;
      return;
    }
  }
  const float a0 = (float)g[0];
  const float ainv = (float)(n - 1) / ((float)g[n - 1] - a0);
  if (std::isfinite(ainv) && worst(vh::GRID_LIN, a0, ainv) <= 2.f) {
    *mode = vh::GRID_LIN;
    *x0 = a0;
    *inv = ainv;
  }
}

namespace vh {
const char* eos_problem(const vh_eos& e) {
  auto size_ok = [](int ne, int nn) { return ne >= 2 && nn >= 2 && (long long)ne * nn <= (1LL << 30); };
  switch (e.kind) {
    case VH_EOS_CONFORMAL:
      return nullptr;
    case VH_EOS_TABLE:
      if (!size_ok(e.ne, e.nn))
        return "EoS table needs ne >= 2, nn >= 2 and at most 2^30 points";
      if (!e.egrid || !e.ngrid || !e.p || !e.T || !e.mub) return "EoS table needs all five arrays";
      return nullptr;
    case VH_EOS_TABLE3:
      if (e.ne < 2 || e.nn < 2 || (long long)e.ne * e.nn * e.nn * e.nn > (1LL << 31))
        return "EoS3f table needs ne >= 2, nn >= 2 and at most 2^31 points";
      if (!e.egrid || !e.ngrid || !e.p || !e.T || !e.mub || !e.muq || !e.mus)
        return "EoS3f table needs all seven arrays";
      return nullptr;
    case VH_EOS_AZH: {
      const vh_eos::vh_eos_azh::vh_eos_azh_table* t[6] = {&e.azh.p1, &e.azh.p2, &e.azh.T1,
                                                          &e.azh.T2, &e.azh.mu1, &e.azh.mu2};
      for (auto* x : t) {
        if (!size_ok(x->ne, x->nn) || !x->v)
          return "EoSAZH tables need ne >= 2, nn >= 2, at most 2^30 points and their values";
        if (!(x->de > 0.) || !(x->dn > 0.) || !(x->emin > 0.))
          return "EoSAZH tables need de > 0, dn > 0 and emin > 0";
      }
      return nullptr;
    }
    case VH_EOS_SMASH: {
      const vh_eos::vh_eos_smash& h = e.smash;
      if (h.ne < 2 || h.nnb < 2 || h.nnq < 2 || (long long)h.ne * h.nnb * h.nnq > (1LL << 31))
        return "EoSSmash table needs ne, nnb, nnq >= 2 and at most 2^31 points";
      if (!h.p || !h.T || !h.mub || !h.muq || !h.mus) return "EoSSmash table needs all five arrays";
      if (!(h.emin < h.emax) || !(h.nbmin < h.nbmax) || !(h.nqmin < h.nqmax))
        return "EoSSmash table needs emin < emax, nbmin < nbmax, nqmin < nqmax";
      return nullptr;
    }
    case VH_EOS_HADRON: {
      const vh_eos::vh_eos_hadron& h = e.hadron;
      if (h.ne < 2 || h.nnb < 2 || h.nnq < 2 || (long long)h.ne * h.nnb * h.nnq > (1LL << 31))
        return "EoSHadron table needs ne, nnb, nnq >= 2 and at most 2^31 points";
      if (!h.p || !h.T || !h.mub || !h.muq || !h.mus || !h.status)
        return "EoSHadron table needs all six arrays";
      if (!(h.e0 > 0.) || !(h.n0 > 0.) || !(h.logemin < h.logemax) || !(h.lognmax > 0.))
        return "EoSHadron table needs e0, n0 > 0, logemin < logemax and lognmax > 0";
      return nullptr;
    }
    case VH_EOS_CHIRAL:
    case VH_EOS_CMFE:
      for (const vh_eos_aux& x : e.aux) {
        if (!size_ok(x.ne, x.nn) || !x.p || !x.T || !x.mub || !x.mus)
          return "chiral EoS table missing, smaller than 2 x 2 or above 2^30 points";
        // the uniform grids' steps (emax - emin) / (ne - 1) divide the lookups
        if (!(x.emin < x.emax) || !(x.nmin < x.nmax) || !std::isfinite(x.emax - x.emin) ||
            !std::isfinite(x.nmax - x.nmin))
          return "chiral EoS table needs finite emin < emax and nmin < nmax";
      }
      return nullptr;
    default:
      return "unsupported EoS kind (no device lowering)";
  }
}
}  // namespace vh

extern "C" {

int vh_abi_version(void) { return VH_ABI_VERSION; }

const char* vh_last_error(vh_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

vh_status vh_destroy(vh_ctx* ctx) {
  if (!ctx) return VH_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->surf_stream) {
    cudaStreamSynchronize(ctx->surf_stream);
    cudaStreamDestroy(ctx->surf_stream);
  }
  if (ctx->snap_ev) cudaEventDestroy(ctx->snap_ev);
  for (cudaGraphExec_t& x : ctx->step_exec)
    if (x) cudaGraphExecDestroy(x);
  for (cudaGraphExec_t& x : ctx->host_exec)
    if (x) cudaGraphExecDestroy(x);
  if (ctx->copy_up) cudaStreamDestroy(ctx->copy_up);
  if (ctx->copy_down) cudaStreamDestroy(ctx->copy_down);
  for (cudaEvent_t e : ctx->host_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->surf.host) cudaFreeHost(ctx->surf.host);
  for (cudaEvent_t e : ctx->evpool) cudaEventDestroy(e);
  if (ctx->surf_ev) cudaEventDestroy(ctx->surf_ev);
  if (ctx->t0) cudaEventDestroy(ctx->t0);
  if (ctx->t1) cudaEventDestroy(ctx->t1);
  delete ctx;
  return VH_OK;
}

// Lowers an EoS descriptor into device tables (allocated on the
// context, freed with it): the hydro EoS at vh_create, the surface EoS at
// vh_set_surface_eos.
static vh_status upload_eos(vh_ctx* c, const vh_eos* eos, vh::EosDev& E) {
  vh_status st = VH_OK;
  cudaError_t e = cudaSuccess;
  (void)e;
  E.kind = eos->kind;
  E.conf_cnst = eos->conf_cnst;
  E.tol = 0.00001;  // src/rmn.cpp:96
  E.vguess = nullptr;
  E.stats = nullptr;
  E.slope = 0;  // the reference's constant dp/de (src/rmn.cpp:36)
  if (eos->kind == VH_EOS_TABLE) {
    const int ne = eos->ne, nn = eos->nn;
    double* buf = nullptr;
    if ((st = dalloc(c, &buf, (size_t)((size_t)ne + nn + 3 * (size_t)ne * nn + (size_t)(ne - 1) + (nn - 1)))) != VH_OK) return st;
    E.ne = ne;
    E.nn = nn;
    choose_axis_mode(eos->egrid, ne, &E.emode, &E.e0, &E.einv);
    choose_axis_mode(eos->ngrid, nn, &E.nmode, &E.n0, &E.ninv);
    E.egrid = buf;
    E.ngrid = buf + ne;
    E.p = buf + ne + nn;
    E.T = E.p + (size_t)ne * nn;
    E.mub = E.T + (size_t)ne * nn;
    const size_t tb = (size_t)ne * nn * sizeof(double);
    if ((e = cudaMemcpy((void*)E.egrid, eos->egrid, ne * sizeof(double), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy((void*)E.ngrid, eos->ngrid, nn * sizeof(double), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy((void*)E.p, eos->p, tb, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy((void*)E.T, eos->T, tb, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy((void*)E.mub, eos->mub, tb, cudaMemcpyHostToDevice))) {
      cuda_fail(c, e, "vh_create: EoS upload");
      return VH_ERR_CUDA;
    }
    // reciprocals of the axis intervals for the interpolation weights
    // (vh::interp_weight); an axis with an interval out of crm::mk_div's
    // range keeps the divide
    double* rdev = buf + ne + nn + 3 * (size_t)ne * nn;
    const double* axes[2] = {eos->egrid, eos->ngrid};
    const int lens[2] = {ne, nn};
    E.erinv = E.nrinv = nullptr;
    for (int a = 0; a < 2; a++) {
      std::vector<double> r((size_t)lens[a] - 1);
      bool ok = true;
      for (int k = 0; k + 1 < lens[a]; k++) {
        const double den = axes[a][k + 1] - axes[a][k];
        ok = ok && vh::crm::mk_den_ok(den);
        r[k] = 1.0 / den;
      }
      if (ok) {
        if ((e = cudaMemcpy(rdev, r.data(), r.size() * sizeof(double), cudaMemcpyHostToDevice))) {
          cuda_fail(c, e, "vh_create: EoS upload");
          return VH_ERR_CUDA;
        }
        (a == 0 ? E.erinv : E.nrinv) = rdev;
      }
      rdev += r.size();
    }
  }
  if (eos->kind == VH_EOS_TABLE3) {
    const int ne = eos->ne, nn = eos->nn;
    const size_t n = (size_t)ne * nn * nn * nn;
    double* buf = nullptr;
    if ((st = dalloc(c, &buf, (size_t)((size_t)ne + nn + 5 * n))) != VH_OK) return st;
    E.ne = ne;
    E.nn = nn;
    E.emode = E.nmode = vh::GRID_BSEARCH;
    E.erinv = E.nrinv = nullptr;
    E.egrid = buf;
    E.ngrid = buf + ne;
    double* t = buf + ne + nn;
    const double* src[5] = {eos->p, eos->T, eos->mub, eos->muq, eos->mus};
    e = cudaMemcpy(buf, eos->egrid, ne * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(buf + ne, eos->ngrid, nn * sizeof(double), cudaMemcpyHostToDevice);
    for (int q = 0; q < 5 && e == cudaSuccess; q++)
      e = cudaMemcpy(t + q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cuda_fail(c, e, "vh_create: EoS upload");
      return VH_ERR_CUDA;
    }
    E.p = t;
    E.T = t + n;
    E.mub = t + 2 * n;
    E.muq = t + 3 * n;
    E.mus = t + 4 * n;
    // EoS3f::getun (src/eo3.cpp:115-130) of a zero charge: every lookup's
    // nq and ns
    int k1 = 0, k2 = nn - 1;
    while (k2 - k1 > 1) {
      const int k = (k1 + k2) / 2;
      if (0. < eos->ngrid[k])
        k2 = k;
      else
        k1 = k;
    }
    int ix = k1 > nn - 2 ? nn - 2 : k1;
    if (ix < 0) ix = 0;
    E.iq0 = ix;
    E.uq0 = (0. - eos->ngrid[k1]) / (eos->ngrid[k2] - eos->ngrid[k1]);
  }
  if (eos->kind == VH_EOS_CHIRAL || eos->kind == VH_EOS_CMFE) {
    for (int k = 0; k < 2; k++) {
      const vh_eos_aux& x = eos->aux[k];
      const size_t n = (size_t)x.ne * x.nn;
      double* buf = nullptr;
      if ((st = dalloc(c, &buf, (size_t)(4 * n))) != VH_OK) return st;
      const double* src[4] = {x.p, x.T, x.mub, x.mus};
      for (int q = 0; q < 4; q++)
        if ((e = cudaMemcpy(buf + q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice))) {
          cuda_fail(c, e, "vh_create: EoS upload");
          return VH_ERR_CUDA;
        }
      E.ch[k] = vh::ChiralAux{x.ne, x.nn, x.emin, x.emax, x.nmin, x.nmax,
                                   buf, buf + n, buf + 2 * n, buf + 3 * n};
    }
  }
  if (eos->kind == VH_EOS_AZH) {
    const vh_eos::vh_eos_azh::vh_eos_azh_table* t[6] = {
        &eos->azh.p1, &eos->azh.p2, &eos->azh.T1, &eos->azh.T2, &eos->azh.mu1, &eos->azh.mu2};
    size_t n = 0;
    for (auto* x : t) n += (size_t)x->ne * x->nn;
    double* buf = nullptr;
    if ((st = dalloc(c, &buf, n)) != VH_OK) return st;
    e = cudaSuccess;
    size_t off = 0;
    for (int q = 0; q < 6; q++) {
      const size_t m = (size_t)t[q]->ne * t[q]->nn;
      if (e == cudaSuccess)
        e = cudaMemcpy(buf + off, t[q]->v, m * sizeof(double), cudaMemcpyHostToDevice);
      E.az[q] = vh::AzhTab{t[q]->ne, t[q]->nn, t[q]->emin, t[q]->nmin, t[q]->de, t[q]->dn, buf + off};
      off += m;
    }
    if (e != cudaSuccess) {
      cuda_fail(c, e, "EoS upload");
      return VH_ERR_CUDA;
    }
  }
  if (eos->kind == VH_EOS_SMASH) {
    const vh_eos::vh_eos_smash& h = eos->smash;
    vh::SmashTab& H = E.sm;
    H.ne = h.ne;
    H.nnb = h.nnb;
    H.nnq = h.nnq;
    H.emin = h.emin;
    H.emax = h.emax;
    H.nbmin = h.nbmin;
    H.nbmax = h.nbmax;
    H.nqmin = h.nqmin;
    H.nqmax = h.nqmax;
    const size_t n = (size_t)h.ne * h.nnb * h.nnq;
    double* buf = nullptr;
    if ((st = dalloc(c, &buf, 5 * n)) != VH_OK) return st;
    const double* src[5] = {h.p, h.T, h.mub, h.muq, h.mus};
    e = cudaSuccess;
    for (int q = 0; q < 5 && e == cudaSuccess; q++)
      e = cudaMemcpy(buf + q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cuda_fail(c, e, "EoS upload");
      return VH_ERR_CUDA;
    }
    H.p = buf;
    H.T = buf + n;
    H.mub = buf + 2 * n;
    H.muq = buf + 3 * n;
    H.mus = buf + 4 * n;
  }
  if (eos->kind == VH_EOS_HADRON) {
    const vh_eos::vh_eos_hadron& h = eos->hadron;
    vh::HadronTab& H = E.h;
    H.ne = h.ne;
    H.nnb = h.nnb;
    H.nnq = h.nnq;
    H.e0 = h.e0;
    H.n0 = h.n0;
    H.logemin = h.logemin;
    H.logemax = h.logemax;
    H.lognmax = h.lognmax;
    // the constructor's derived constants (src/eoHadron.cpp:49-53)
    const double dxnb = (2.0 * h.lognmax) / (h.nnb - 1);
    const double dxnq = (2.0 * h.lognmax) / (h.nnq - 1);
    H.nb_abs_min = h.n0 * exp(2.0 * dxnb - h.lognmax);
    H.nq_abs_min = h.n0 * exp(2.0 * dxnq - h.lognmax);
    H.e_min = h.e0 * exp(h.logemin);
    const size_t n = (size_t)h.ne * h.nnb * h.nnq;
    double* buf = nullptr;
    int* sbuf = nullptr;
    if ((st = dalloc(c, &buf, 5 * n)) != VH_OK) return st;
    if ((st = dalloc(c, &sbuf, n)) != VH_OK) return st;
    const double* src[5] = {h.p, h.T, h.mub, h.muq, h.mus};
    e = cudaSuccess;
    for (int q = 0; q < 5 && e == cudaSuccess; q++)
      e = cudaMemcpy(buf + q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(sbuf, h.status, n * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cuda_fail(c, e, "EoS upload");
      return VH_ERR_CUDA;
    }
    H.p = buf;
    H.T = buf + n;
    H.mub = buf + 2 * n;
    H.muq = buf + 3 * n;
    H.mus = buf + 4 * n;
    H.status = sbuf;
  }
  return VH_OK;
}

// The EoS outputSurface / outputCorona run with (Fluid's eosH, swapped in
// for their whole body, src/fld.cpp:540-542, 870-872), with the hydro
// EoS's root-find settings.
static vh::EosDev surf_eos(const vh_ctx* c) {
  vh::EosDev E = c->has_eosH ? c->eosH : c->eos;
  E.tol = c->eos.tol;
  E.stats = c->eos.stats;
  E.vguess = nullptr;
  E.slope = 0;
  return E;
}

vh_status vh_create(const vh_grid* grid, const vh_eos* eos, const vh_trcoeff* tr, double tau0,
                    double dt, int device, vh_ctx** out) {
  if (!out) return fail(nullptr, VH_ERR_ARG, "vh_create: out is NULL");
  *out = nullptr;
  if (!grid || !eos || !tr) return fail(nullptr, VH_ERR_ARG, "vh_create: NULL argument");
  if (grid->nx < 2 || grid->ny < 2 || grid->nz < 1)
    return fail(nullptr, VH_ERR_ARG, "vh_create: need nx >= 2, ny >= 2, nz >= 1");
  // src/main.cpp:153-155 (checkGridBorders) requires min < max on every axis
  if (!(grid->xmin < grid->xmax) || !(grid->ymin < grid->ymax) || !(grid->etamin < grid->etamax))
    return fail(nullptr, VH_ERR_ARG, "vh_create: the grid needs min < max on every axis");
  if (!(tau0 > 0.)) return fail(nullptr, VH_ERR_ARG, "vh_create: tau0 must be positive");
  if (const char* why = vh::eos_problem(*eos))
    return fail(nullptr, VH_ERR_ARG, std::string("vh_create: ") + why);
  if (eos->kind == VH_EOS_HADRON || eos->kind == VH_EOS_SMASH)
    return fail(nullptr, VH_ERR_ARG,
                "vh_create: EoSHadron / EoSSmash are surface EoS (vh_set_surface_eos)");
  const double dx = (grid->xmax - grid->xmin) / (grid->nx - 1);
  const double dy = (grid->ymax - grid->ymin) / (grid->ny - 1);
  if (!(dt > 0.) || dt > dx / 2. || dt > dy / 2.)
    return fail(nullptr, VH_ERR_ARG, "vh_create: too big delta_tau (dt > dx/2 or dy/2)");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, VH_ERR_CUDA, std::string("vh_create: no CUDA device: ") +
                                          (e != cudaSuccess ? cudaGetErrorString(e) : "count 0"));
  if (device < 0 || device >= ndev) return fail(nullptr, VH_ERR_ARG, "vh_create: bad device index");

  vh_ctx* c = new vh_ctx;
  c->err.clear();
  c->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess) {
    g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    delete c;
    return VH_ERR_CUDA;
  }
  auto bail = [&](vh_status st) {
    g_create_error = c->err;
    vh_destroy(c);
    return st;
  };
  if ((e = vh::step_kernels_setup()) != cudaSuccess) {
    cuda_fail(c, e, "vh_create: kernel attributes");
    return bail(VH_ERR_CUDA);
  }
  vh::Geo& g = c->g;
  g.nx = grid->nx;
  g.ny = grid->ny;
  g.nz = grid->nz;
  g.N = (long long)grid->nx * grid->ny * grid->nz;
  g.dx = dx;
  g.dy = dy;
  g.dz = grid->dz > 0. ? grid->dz : (grid->etamax - grid->etamin) / (grid->nz - 1);
  vh::geo_whole(g);
  c->grid = *grid;
  c->tau = tau0;
  c->dt = dt;
  c->fluid_dt = dt;
  c->tr = vh::TrDev{tr->etaS0, tr->zetaS0, tr->ah, tr->al, tr->aRho, tr->T0, tr->etaSMin,
                    tr->etaSEpsilonMin, tr->etaSShiftMuB, tr->etaSScaleMuB,
                    tr->zetaSPeakEpsilon, tr->zetaSScaleBeta, tr->zetaSSigmaMinus,
                    tr->zetaSSigmaPlus, tr->etaSparam, tr->zetaSparam, tr->zetaSPeakT,
                    tr->zetaSWidthT};
  // TransportCoeff::isViscous, src/trancoeff.h:39-45
  c->viscous = tr->etaS0 > 0. || tr->zetaS0 > 0. || tr->etaSparam > 0 || tr->zetaSparam > 0;

  const long long N = g.N;
  vh::Fields& f = c->f;
  vh_status st = VH_OK;
#define ALLOC(p, n) \
  if ((st = dalloc(c, &(p), (size_t)(n))) != VH_OK) return bail(st)
  ALLOC(f.Q, 7 * N);
  ALLOC(f.Qh, 7 * N);
  ALLOC(f.Qprev, 7 * N);
  ALLOC(f.pi, 10 * N);
  ALLOC(f.piH, 10 * N);
  ALLOC(f.Pi, N);
  ALLOC(f.PiH, N);
  ALLOC(f.vcc, N);
  ALLOC(f.m, 3 * N);
  ALLOC(f.m2, 3 * N);
  c->m_first = f.m;
  ALLOC(f.Fx, 7 * N);
  ALLOC(f.Fy, 7 * N);
  ALLOC(f.Fz, 7 * N);
  if (c->viscous) {
    ALLOC(f.flux, 4 * N);
    ALLOC(f.pA, 8 * N);
    ALLOC(f.pD, 4 * N);
    ALLOC(f.pTh, 9 * N);
    ALLOC(f.pBC, 9 * N);
    ALLOC(f.pi0, 10 * N);
    ALLOC(f.piH0, 10 * N);
    ALLOC(f.Pi0, N);
    ALLOC(f.PiH0, N);
    ALLOC(f.active, N);
    ALLOC(f.nactive, 1);
  }
  ALLOC(c->clk, 2);
  ALLOC(c->tot_partial, (size_t)vh::totals_blocks(g) * vh::kTotals);
  ALLOC(c->tot_out, vh::kTotals);
  const int ng = g.nx + g.ny + g.nz;
  ALLOC(f.gsrc, ng);
  ALLOC(f.gdst, ng);
  ALLOC(f.err, 1);
  std::vector<int> hsrc(ng);
  std::vector<unsigned char> hdst(ng);
  ghost_map(g.nx, hsrc.data(), hdst.data());
  ghost_map(g.ny, hsrc.data() + g.nx, hdst.data() + g.nx);
  ghost_map(g.nz, hsrc.data() + g.nx + g.ny, hdst.data() + g.nx + g.ny);
  if ((e = cudaMemcpy(f.gsrc, hsrc.data(), ng * sizeof(int), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(f.gdst, hdst.data(), ng, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(f.err, 0, sizeof(unsigned))) ||
      (e = cudaMemcpy(c->clk, std::vector<double>{tau0, dt}.data(), 2 * sizeof(double),
                      cudaMemcpyHostToDevice))) {
    cuda_fail(c, e, "vh_create: upload");
    return bail(VH_ERR_CUDA);
  }
  {
    vh_status se = upload_eos(c, eos, c->eos);
    if (se != VH_OK) return bail(se);
  }
#undef ALLOC
  *out = c;
  return VH_OK;
}

vh_status vh_set_surface_eos(vh_ctx* ctx, const vh_eos* eos) {
  if (!ctx) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_set_surface_eos");
  if (!eos) {
    ctx->has_eosH = false;
    return VH_OK;
  }
  if (eos->kind == VH_EOS_CONFORMAL)
    return fail(ctx, VH_ERR_ARG, "vh_set_surface_eos: the conformal gas is not a surface EoS");
  if (const char* why = vh::eos_problem(*eos))
    return fail(ctx, VH_ERR_ARG, std::string("vh_set_surface_eos: ") + why);
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::EosDev E{};
  vh_status st = upload_eos(ctx, eos, E);
  if (st != VH_OK) return st;
  ctx->eosH = E;
  ctx->has_eosH = true;
  return VH_OK;
}

vh_status vh_set_stream(vh_ctx* ctx, void* stream) {
  if (!ctx) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_set_stream");
  ctx->stream = static_cast<cudaStream_t>(stream);
  return VH_OK;
}

struct FieldSpec {
  double* vh_state_view::*host;
  double* vh::Fields::*dev;
  int ncomp;
};

static const FieldSpec kFields[] = {
    {&vh_state_view::Q, &vh::Fields::Q, 7},       {&vh_state_view::Qh, &vh::Fields::Qh, 7},
    {&vh_state_view::Qprev, &vh::Fields::Qprev, 7}, {&vh_state_view::pi, &vh::Fields::pi, 10},
    {&vh_state_view::piH, &vh::Fields::piH, 10},  {&vh_state_view::Pi, &vh::Fields::Pi, 1},
    {&vh_state_view::PiH, &vh::Fields::PiH, 1},   {&vh_state_view::m, &vh::Fields::m, 3},
    {&vh_state_view::viscCorrCut, &vh::Fields::vcc, 1},
};

vh_status vh_upload_async(vh_ctx* ctx, const vh_state_view* h) {
  if (!ctx || !h) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_upload_async");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  for (const FieldSpec& fs : kFields) {
    const double* src = h->*(fs.host);
    if (!src) continue;
    VH_CUDA(ctx, cudaMemcpyAsync(ctx->f.*(fs.dev), src, sizeof(double) * fs.ncomp * ctx->g.N,
                                 cudaMemcpyHostToDevice, ctx->stream));
  }
  ctx->uploaded = true;
  return VH_OK;
}

vh_status vh_download_async(vh_ctx* ctx, const vh_state_view* h) {
  if (!ctx || !h) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  for (const FieldSpec& fs : kFields) {
    double* dst = h->*(fs.host);
    if (!dst) continue;
    VH_CUDA(ctx, cudaMemcpyAsync(dst, ctx->f.*(fs.dev), sizeof(double) * fs.ncomp * ctx->g.N,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  }
  return VH_OK;
}

vh_status vh_upload_state(vh_ctx* ctx, const vh_state_view* h) {
  if (!ctx || !h) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_upload_state");
  if (!h->Q) return fail(ctx, VH_ERR_ARG, "vh_upload_state: Q is required");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  const long long N = ctx->g.N;
  vh::Fields& f = ctx->f;
  cudaStream_t s = ctx->stream;
  vh_status st = vh_upload_async(ctx, h);
  if (st != VH_OK) return st;
  vh::launch_zero_negative_rows(f.Q, N, s);  // Cell::setQ
  if (!h->Qprev)
    VH_CUDA(ctx, cudaMemcpyAsync(f.Qprev, f.Q, 7 * N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (!h->Qh) VH_CUDA(ctx, cudaMemsetAsync(f.Qh, 0, 7 * N * sizeof(double), s));
  if (!h->pi) VH_CUDA(ctx, cudaMemsetAsync(f.pi, 0, 10 * N * sizeof(double), s));
  if (!h->piH) VH_CUDA(ctx, cudaMemsetAsync(f.piH, 0, 10 * N * sizeof(double), s));
  if (!h->Pi) VH_CUDA(ctx, cudaMemsetAsync(f.Pi, 0, N * sizeof(double), s));
  if (!h->PiH) VH_CUDA(ctx, cudaMemsetAsync(f.PiH, 0, N * sizeof(double), s));
  if (!h->m) VH_CUDA(ctx, cudaMemsetAsync(f.m, 0, 3 * N * sizeof(double), s));
  if (!h->viscCorrCut) vh::launch_fill(f.vcc, N, 1.0, s);
  VH_CUDA(ctx, cudaGetLastError());
  VH_CUDA(ctx, cudaStreamSynchronize(s));
  return VH_OK;
}

vh_status vh_download_state(vh_ctx* ctx, const vh_state_view* h) {
  vh_status st = vh_download_async(ctx, h);
  if (st != VH_OK) return st;
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VH_OK;
}

static vh_status planes(vh_ctx* ctx, int z0, int nplanes, double* buf, bool pack,
                        const char* who) {
  if (!ctx || !buf || nplanes < 0) return VH_ERR_ARG;
  if (z0 < 0 || (long long)z0 + nplanes > ctx->g.nz)
    return fail(ctx, VH_ERR_ARG, std::string(who) + ": planes outside the grid's z range");
  if (!pack) VH_NOT_PENDING(ctx, "vh_unpack_planes");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::PlaneFields pf{};
  int k = 0;
  for (const FieldSpec& fs : kFields) {
    pf.p[k] = ctx->f.*(fs.dev);
    pf.ncomp[k] = fs.ncomp;
    pf.ncomp_total += fs.ncomp;
    k++;
  }
  pf.nfield = k;
  const long long nxy = (long long)ctx->g.nx * ctx->g.ny;
  vh::launch_planes(pf, ctx->g.N, nxy, z0, nplanes, buf, pack, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  return VH_OK;
}

vh_status vh_pack_planes(vh_ctx* ctx, int z0, int nplanes, double* buf_dev) {
  return planes(ctx, z0, nplanes, buf_dev, true, "vh_pack_planes");
}

vh_status vh_unpack_planes(vh_ctx* ctx, int z0, int nplanes, const double* buf_dev) {
  return planes(ctx, z0, nplanes, const_cast<double*>(buf_dev), false, "vh_unpack_planes");
}

vh_status vh_device_state(vh_ctx* ctx, vh_state_view* d) {
  if (!ctx || !d) return VH_ERR_ARG;
  for (const FieldSpec& fs : kFields) d->*(fs.host) = ctx->f.*(fs.dev);
  return VH_OK;
}

static vh::StepArgs step_args(vh_ctx* ctx) {
  vh::StepArgs a;
  a.g = ctx->g;
  a.eos = ctx->eos;
  a.eos.vguess = ctx->mlp ? ctx->vguess : nullptr;
  a.tr = ctx->tr;
  a.f = ctx->f;
  a.clk = ctx->clk;  // holds (tau, dt): set when the host changes them, advanced per step
  a.viscous = ctx->viscous;
  a.vort = ctx->vort_on && ctx->viscous ? &ctx->vort : nullptr;
  return a;
}

// Gives every kernel node of a captured step the device's highest stream
// priority, so that a pipelined surface pass on its own stream (priority 0)
// takes only the SM room the step's kernels leave between them.
static cudaError_t graph_high_priority(cudaGraph_t graph) {
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  size_t n = 0;
  if (e == cudaSuccess) e = cudaGraphGetNodes(graph, nullptr, &n);
  std::vector<cudaGraphNode_t> nodes(n);
  if (e == cudaSuccess && n) e = cudaGraphGetNodes(graph, nodes.data(), &n);
  for (size_t i = 0; e == cudaSuccess && i < n; i++) {
    cudaGraphNodeType t;
    if ((e = cudaGraphNodeGetType(nodes[i], &t)) != cudaSuccess || t != cudaGraphNodeTypeKernel)
      continue;
    cudaLaunchAttributeValue v = {};
    v.priority = greatest;
    e = cudaGraphKernelNodeSetAttribute(nodes[i], cudaLaunchAttributePriority, &v);
  }
  return e;
}

// One step (the learned guess, performStep, tau += dt on the device clock)
// captured into ctx->step_exec[par]; false if the capture is refused.
static bool capture_step(vh_ctx* ctx, int par) {
  if (!ctx->cap_stream &&
      cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (ctx->step_exec[par]) {
    cudaGraphExecDestroy(ctx->step_exec[par]);
    ctx->step_exec[par] = nullptr;
  }
  const vh::StepArgs a = step_args(ctx);
  cudaStream_t s = ctx->cap_stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (ctx->mlp) vh::launch_mlp_guess(ctx->mlp->packed, ctx->f.Q, ctx->g.N, ctx->clk, ctx->vguess, s);
  const int n = vh::launch_step(a, s);
  vh::launch_clock_op(ctx->clk, 0, 0, s);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  unsigned long long flags = cudaGraphInstantiateFlagUseNodePriority;
  if (e == cudaSuccess && graph_high_priority(graph) != cudaSuccess) {
    cudaGetLastError();  // the step runs at its stream's priority then
    flags = 0;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->step_exec[par], graph, flags);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->step_exec[par] = nullptr;
    return false;
  }
  ctx->step_version[par] = ctx->version;
  ctx->step_launches[par] = n;
  return true;
}

vh_status vh_step(vh_ctx* ctx) {
  if (!ctx) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_step: no state uploaded");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->prof && ctx->step_graphs) {
    const int par = ctx->f.m == ctx->m_first ? 0 : 1;
    if ((ctx->step_exec[par] && ctx->step_version[par] == ctx->version) ||
        capture_step(ctx, par)) {
      VH_CUDA(ctx, cudaGraphLaunch(ctx->step_exec[par], ctx->stream));
      ctx->launches = ctx->step_launches[par];
      std::swap(ctx->f.m, ctx->f.m2);
      ctx->tau += ctx->dt;  // src/hdo.cpp:1095
      return VH_OK;
    }
    ctx->step_graphs = false;  // launch directly from now on
  }
  const vh::StepArgs a = step_args(ctx);
  if (ctx->mlp)  // start points for this step's root finds from Q at tau
    vh::launch_mlp_guess(ctx->mlp->packed, ctx->f.Q, ctx->g.N, ctx->clk, ctx->vguess, ctx->stream);
  if (ctx->prof) {
    EventMarker mk(ctx, 0);
    mk.after(-1);  // start event of this step
    mk.prev = ctx->segs.back().ev1;
    ctx->segs.pop_back();
    ctx->launches = vh::launch_step(a, ctx->stream, &mk);
    if (mk.err != cudaSuccess) return cuda_fail(ctx, mk.err, "vh_step: profiling event");
  } else {
    ctx->launches = vh::launch_step(a, ctx->stream);
  }
  vh::launch_clock_op(ctx->clk, 0, 0, ctx->stream);  // tau += dt on the device
  VH_CUDA(ctx, cudaGetLastError());
  std::swap(ctx->f.m, ctx->f.m2);
  ctx->tau += ctx->dt;  // src/hdo.cpp:1095
  return VH_OK;
}

// vh_step_host's copies hung on the step's kernels: m back once updateM
// has run, the viscous inputs awaited before the first kernel after the
// corrector's update (the ghost copy, which reads pi and Pi), piH, PiH and
// viscCorrCut back once the relaxation's advection (their last writer) ran
struct HostCopyMarker : vh::LaunchMarker {
  vh_ctx* ctx;
  cudaStream_t s;
  const vh_state_view* out;
  int nupdate = 0;
  bool advected = false;
  cudaError_t err = cudaSuccess;
  HostCopyMarker(vh_ctx* c, cudaStream_t st, const vh_state_view* o) : ctx(c), s(st), out(o) {}
  void down(double* dst, const double* src, int ncomp) {
    if (dst && err == cudaSuccess)
      err = cudaMemcpyAsync(dst, src, sizeof(double) * ncomp * ctx->g.N, cudaMemcpyDeviceToHost,
                            ctx->copy_down);
  }
  void fork_down(cudaEvent_t ev) {
    if (err == cudaSuccess) err = cudaEventRecord(ev, s);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(ctx->copy_down, ev, 0);
  }
  void after(int kind) override {
    if (err != cudaSuccess) return;
    if (kind == vh::KK_UPDATE_M) {
      if (out->m) {
        fork_down(ctx->host_ev[2]);
        down(out->m, ctx->f.m2, 3);  // the next step's fill fractions
      }
    } else if (kind == vh::KK_UPDATE && ++nupdate == 2) {
      err = cudaStreamWaitEvent(s, ctx->host_ev[1], 0);
    } else if (kind == vh::KK_IS_ADVECT) {
      advected = true;
      if (out->piH || out->PiH || out->viscCorrCut) {
        fork_down(ctx->host_ev[3]);
        down(out->piH, ctx->f.piH, 10);
        down(out->PiH, ctx->f.PiH, 1);
        down(out->viscCorrCut, ctx->f.vcc, 1);
      }
    }
  }
};

static std::vector<const void*> host_key(const vh_state_view* in, const vh_state_view* out) {
  std::vector<const void*> k;
  for (const FieldSpec& fs : kFields) {
    k.push_back(in->*(fs.host));
    k.push_back(out->*(fs.host));
  }
  return k;
}

// The step with its host copies captured into ctx->host_exec[par]; false if
// the capture is refused (pageable host memory may be, for one).
static bool capture_host_step(vh_ctx* ctx, int par, const vh_state_view* in,
                              const vh_state_view* out) {
  cudaError_t e = cudaSuccess;
  if (!ctx->cap_stream) e = cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess && !ctx->copy_up)
    e = cudaStreamCreateWithFlags(&ctx->copy_up, cudaStreamNonBlocking);
  if (e == cudaSuccess && !ctx->copy_down)
    e = cudaStreamCreateWithFlags(&ctx->copy_down, cudaStreamNonBlocking);
  for (cudaEvent_t& ev : ctx->host_ev)
    if (e == cudaSuccess && !ev) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (ctx->host_exec[par]) {
    cudaGraphExecDestroy(ctx->host_exec[par]);
    ctx->host_exec[par] = nullptr;
  }
  const vh::StepArgs a = step_args(ctx);
  const vh::Fields& F = ctx->f;
  const long long N = ctx->g.N;
  cudaStream_t s = ctx->cap_stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  auto copy = [&](double* dst, const double* src, int ncomp, cudaMemcpyKind kind, cudaStream_t st) {
    if (src && dst && e == cudaSuccess)
      e = cudaMemcpyAsync(dst, src, sizeof(double) * ncomp * N, kind, st);
  };
  // what the ideal stages read goes up first, on the step's stream
  copy(F.Q, in->Q, 7, cudaMemcpyHostToDevice, s);
  copy(F.m, in->m, 3, cudaMemcpyHostToDevice, s);
  copy(F.Qh, in->Qh, 7, cudaMemcpyHostToDevice, s);
  copy(F.Qprev, in->Qprev, 7, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->host_ev[0], s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_up, ctx->host_ev[0], 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_down, ctx->host_ev[0], 0);
  // the viscous inputs beside the ideal stages
  copy(F.pi, in->pi, 10, cudaMemcpyHostToDevice, ctx->copy_up);
  copy(F.piH, in->piH, 10, cudaMemcpyHostToDevice, ctx->copy_up);
  copy(F.Pi, in->Pi, 1, cudaMemcpyHostToDevice, ctx->copy_up);
  copy(F.PiH, in->PiH, 1, cudaMemcpyHostToDevice, ctx->copy_up);
  copy(F.vcc, in->viscCorrCut, 1, cudaMemcpyHostToDevice, ctx->copy_up);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->host_ev[1], ctx->copy_up);
  HostCopyMarker mk(ctx, s, out);
  int n = 0;
  if (e == cudaSuccess) {
    if (ctx->mlp) vh::launch_mlp_guess(ctx->mlp->packed, F.Q, N, ctx->clk, ctx->vguess, s);
    n = vh::launch_step(a, s, &mk);
    vh::launch_clock_op(ctx->clk, 0, 0, s);
    e = mk.err;
  }
  // the rest comes back at the end
  copy(out->Q, F.Q, 7, cudaMemcpyDeviceToHost, s);
  copy(out->Qh, F.Qh, 7, cudaMemcpyDeviceToHost, s);
  copy(out->Qprev, F.Qprev, 7, cudaMemcpyDeviceToHost, s);
  copy(out->pi, F.pi, 10, cudaMemcpyDeviceToHost, s);
  copy(out->Pi, F.Pi, 1, cudaMemcpyDeviceToHost, s);
  if (!mk.advected) {
    copy(out->piH, F.piH, 10, cudaMemcpyDeviceToHost, s);
    copy(out->PiH, F.PiH, 1, cudaMemcpyDeviceToHost, s);
    copy(out->viscCorrCut, F.vcc, 1, cudaMemcpyDeviceToHost, s);
  }
  // join the copy streams
  if (e == cudaSuccess) e = cudaEventRecord(ctx->host_ev[4], ctx->copy_down);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->host_ev[4], 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->host_ev[1], 0);
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s, &graph);
  if (e == cudaSuccess) e = ec;
  unsigned long long flags = cudaGraphInstantiateFlagUseNodePriority;
  if (e == cudaSuccess && graph_high_priority(graph) != cudaSuccess) {
    cudaGetLastError();
    flags = 0;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->host_exec[par], graph, flags);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->host_exec[par] = nullptr;
    return false;
  }
  ctx->host_version[par] = ctx->version;
  ctx->host_key[par] = host_key(in, out);
  ctx->step_launches[par] = n;
  return true;
}

vh_status vh_step_host(vh_ctx* ctx, const vh_state_view* in, const vh_state_view* out) {
  if (!ctx || !in || !out) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_step_host");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  if (in->Q) ctx->uploaded = true;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_step_host: no state uploaded");
  if (!ctx->prof && ctx->step_graphs) {
    const int par = ctx->f.m == ctx->m_first ? 0 : 1;
    if ((ctx->host_exec[par] && ctx->host_version[par] == ctx->version &&
         ctx->host_key[par] == host_key(in, out)) ||
        capture_host_step(ctx, par, in, out)) {
      VH_CUDA(ctx, cudaGraphLaunch(ctx->host_exec[par], ctx->stream));
      ctx->launches = ctx->step_launches[par];
      std::swap(ctx->f.m, ctx->f.m2);
      ctx->tau += ctx->dt;  // src/hdo.cpp:1095
      return VH_OK;
    }
  }
  vh_status st = vh_upload_async(ctx, in);
  if (st == VH_OK) st = vh_step(ctx);
  if (st == VH_OK) st = vh_download_async(ctx, out);
  return st;
}

vh_status vh_steps(vh_ctx* ctx, int n) {
  for (int k = 0; k < n; k++) {
    vh_status st = vh_step(ctx);
    if (st != VH_OK) return st;
  }
  return VH_OK;
}

vh_status vh_set_dtau(vh_ctx* ctx, double dt) {
  if (!ctx) return VH_ERR_ARG;
  if (!(dt > 0.) || dt > ctx->g.dx / 2. || dt > ctx->g.dy / 2.)
    return fail(ctx, VH_ERR_ARG, "vh_set_dtau: too big delta_tau (dt > dx/2 or dy/2)");
  ctx->dt = dt;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::launch_clock_set(ctx->clk, ctx->tau, ctx->dt, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  return VH_OK;
}

vh_status vh_get_dtau(vh_ctx* ctx, double* dt) {
  if (!ctx || !dt) return VH_ERR_ARG;
  *dt = ctx->dt;
  return VH_OK;
}

vh_status vh_get_tau(vh_ctx* ctx, double* tau) {
  if (!ctx || !tau) return VH_ERR_ARG;
  *tau = ctx->tau;
  return VH_OK;
}

vh_status vh_set_tau(vh_ctx* ctx, double tau) {
  if (!ctx) return VH_ERR_ARG;
  ctx->tau = tau;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::launch_clock_set(ctx->clk, ctx->tau, ctx->dt, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  return VH_OK;
}

vh_status vh_set_con2prim(vh_ctx* ctx, double tol) {
  if (!ctx) return VH_ERR_ARG;
  if (!(tol > 0.) || !(tol <= 0.00001))
    return fail(ctx, VH_ERR_ARG, "vh_set_con2prim: tol must be in (0, 1e-5]");
  if (ctx->eos.slope && !(tol <= 1e-10))
    return fail(ctx, VH_ERR_ARG,
                "vh_set_con2prim: the table-slope method needs tol <= 1e-10 (set the method "
                "back to VH_C2P_REFERENCE first)");
  ctx->eos.tol = tol;
  ctx->version++;
  return VH_OK;
}

vh_status vh_set_con2prim_method(vh_ctx* ctx, int method) {
  if (!ctx) return VH_ERR_ARG;
  if (method != VH_C2P_REFERENCE && method != VH_C2P_TABLE_SLOPE)
    return fail(ctx, VH_ERR_ARG, "vh_set_con2prim_method: unknown method");
  if (method == VH_C2P_TABLE_SLOPE && (ctx->eos.kind == VH_EOS_TABLE3 || ctx->eos.kind == VH_EOS_AZH ||
                                       ctx->eos.kind == VH_EOS_CMFE))
    return fail(ctx, VH_ERR_ARG,
                "vh_set_con2prim_method: no table slope for the EoS3f, EoSAZH and EoSCMFe kinds");
  if (method == VH_C2P_TABLE_SLOPE && !(ctx->eos.tol <= 1e-10))
    return fail(ctx, VH_ERR_ARG,
                "vh_set_con2prim_method: the table slope needs a tight tolerance "
                "(vh_set_con2prim with tol <= 1e-10 first)");
  ctx->eos.slope = method;
  ctx->version++;
  return VH_OK;
}

vh_status vh_set_con2prim_guess(vh_ctx* ctx, vh_mlp* mlp) {
  if (!ctx) return VH_ERR_ARG;
  if (mlp && mlp->device != ctx->device)
    return fail(ctx, VH_ERR_ARG, "vh_set_con2prim_guess: the network lives on another device");
  if (mlp && !ctx->vguess) {
    VH_CUDA(ctx, cudaSetDevice(ctx->device));
    vh_status st = dalloc(ctx, &ctx->vguess, (size_t)ctx->g.N);
    if (st != VH_OK) return st;
  }
  ctx->mlp = mlp;
  ctx->version++;
  return VH_OK;
}

vh_status vh_mlp_samples(vh_ctx* ctx, float* X, float* Y, long cap, long* n) {
  if (!ctx || cap < 0 || (cap > 0 && (!X || !Y))) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_mlp_samples: no state uploaded");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->ucount) {
    vh_status st = dalloc(ctx, &ctx->ucount, 1);
    if (st != VH_OK) return st;
  }
  VH_CUDA(ctx, cudaMemsetAsync(ctx->ucount, 0, sizeof(unsigned long long), ctx->stream));
  vh::EosDev E = ctx->eos;
  E.tol = 1e-13;  // labels from the root converged to round-off
  E.vguess = nullptr;
  E.slope = 0;
  E.stats = nullptr;
  vh::launch_mlp_samples(E, ctx->f.Q, ctx->g.N, ctx->tau, X, Y, cap, ctx->ucount, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  unsigned long long h = 0;
  VH_CUDA(ctx, cudaMemcpyAsync(&h, ctx->ucount, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (n) *n = (long)std::min<unsigned long long>(h, (unsigned long long)cap);
  return VH_OK;
}

vh_status vh_con2prim_stats(vh_ctx* ctx, int enable, unsigned long long* calls,
                            unsigned long long* iters) {
  if (!ctx) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->c2p_stats) {
    vh_status st = dalloc(ctx, &ctx->c2p_stats, 2);
    if (st != VH_OK) return st;
    VH_CUDA(ctx, cudaMemsetAsync(ctx->c2p_stats, 0, 2 * sizeof(unsigned long long), ctx->stream));
  }
  unsigned long long h[2] = {0, 0};
  VH_CUDA(ctx, cudaMemcpyAsync(h, ctx->c2p_stats, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (calls) *calls = h[0];
  if (iters) *iters = h[1];
  VH_CUDA(ctx, cudaMemsetAsync(ctx->c2p_stats, 0, 2 * sizeof(unsigned long long), ctx->stream));
  ctx->eos.stats = enable ? ctx->c2p_stats : nullptr;
  ctx->version++;
  return VH_OK;
}

vh_status vh_get_grid(vh_ctx* ctx, vh_grid* out) {
  if (!ctx || !out) return VH_ERR_ARG;
  *out = ctx->grid;
  return VH_OK;
}

vh_status vh_advance(vh_ctx* ctx, double dtau, double etamin, double etamax, int nz, int* nsub) {
  if (!ctx) return VH_ERR_ARG;
  int n = 1;
  while (dtau / n > 1.0 * ctx->tau * (etamax - etamin) / (nz - 1)) {
    if (n >= (1 << 30)) return fail(ctx, VH_ERR_ARG, "vh_advance: substep count overflow");
    n *= 2;
  }
  if (nsub) *nsub = n;
  if (n == 1) return vh_step(ctx);
  vh_status st = vh_set_dtau(ctx, ctx->dt / n);
  if (st != VH_OK) return st;
  for (int j = 0; j < n && st == VH_OK; j++) st = vh_step(ctx);
  const vh_status st2 = vh_set_dtau(ctx, ctx->dt * n);
  return st != VH_OK ? st : st2;
}

vh_status vh_resize2x(vh_ctx* ctx, int* resized) {
  if (resized) *resized = 0;
  if (!ctx) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_resize2x: no state uploaded");
  VH_NOT_PENDING(ctx, "vh_resize2x");
  const vh_grid& gr = ctx->grid;
  vh::Geo& g = ctx->g;
  // Fluid::getX / getY / getZ, src/fld.h:62-64
  const double x0 = gr.xmin + 0 * g.dx, x1 = gr.xmin + (g.nx - 1) * g.dx;
  const double y0 = gr.ymin + 0 * g.dy, y1 = gr.ymin + (g.ny - 1) * g.dy;
  if (x0 + x1 > 0.001 || y0 + y1 > 0.001) return VH_OK;
  vh_grid ng = gr;
  ng.dz = 0.;  // the new Fluid derives its cell size from its bounds
  ng.xmin = 2.0 * x0;
  ng.xmax = 2.0 * x1;
  ng.ymin = 2.0 * y0;
  ng.ymax = 2.0 * y1;
  ng.etamin = gr.etamin + 0 * g.dz;
  ng.etamax = gr.etamin + (g.nz - 1) * g.dz;
  // Fluid::Fluid, src/fld.cpp:77-79
  const double ndx = (ng.xmax - ng.xmin) / (g.nx - 1);
  const double ndy = (ng.ymax - ng.ymin) / (g.ny - 1);
  const double ndz = (ng.etamax - ng.etamin) / (g.nz - 1);
  const double dt2 = 2.0 * ctx->dt;
  if (dt2 > ndx / 2. || dt2 > ndy / 2.)
    return fail(ctx, VH_ERR_ARG, "vh_resize2x: too big delta_tau for the resized grid");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->resize_tmp) {
    vh_status st = dalloc(ctx, &ctx->resize_tmp, (size_t)10 * g.N);
    if (st != VH_OK) return st;
  }
  vh::Fields& f = ctx->f;
  struct Plane {
    double* p;
    int n;
  } planes[] = {{f.Q, 7}, {f.Qh, 7}, {f.Qprev, 7}, {f.pi, 10}, {f.piH, 10},
                {f.Pi, 1}, {f.PiH, 1}, {f.m, 3},  {f.vcc, 1}};
  for (const Plane& pl : planes) {
    vh::launch_resize_gather(g, pl.p, ctx->resize_tmp, pl.n, ctx->stream);
    VH_CUDA(ctx, cudaGetLastError());
    VH_CUDA(ctx, cudaMemcpyAsync(pl.p, ctx->resize_tmp, sizeof(double) * pl.n * g.N,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
  }
  ctx->grid = ng;
  g.dx = ndx;
  g.dy = ndy;
  g.dz = ndz;
  ctx->dt = dt2;  // src/main.cpp:268
  vh::launch_clock_set(ctx->clk, ctx->tau, ctx->dt, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  ctx->fluid_dt = dt2;  // the new Fluid's step, src/main.cpp:254-256
  ctx->EtotSurf = ctx->vEff = 0.;  // members of the new Fluid, src/fld.cpp:110-111
  if (ctx->vort.dbeta)  // the new Fluid's cells start from zero (src/main.cpp:257,264-265)
    VH_CUDA(ctx, cudaMemsetAsync(ctx->vort.dbeta, 0, sizeof(double) * 16 * g.N, ctx->stream));
  ctx->version++;
  if (resized) *resized = 1;
  return VH_OK;
}

vh_status vh_active_cells(vh_ctx* ctx, long long* n) {
  if (!ctx || !n) return VH_ERR_ARG;
  *n = 0;
  if (!ctx->f.nactive) return VH_OK;  // an ideal context has no relaxation
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  int h = 0;
  VH_CUDA(ctx, cudaMemcpyAsync(&h, ctx->f.nactive, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *n = h;
  return VH_OK;
}

vh_status vh_error_bits(vh_ctx* ctx, unsigned* bits) {
  if (!ctx || !bits) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  VH_CUDA(ctx, cudaMemcpyAsync(bits, ctx->f.err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                               ctx->stream));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VH_OK;
}

vh_status vh_clear_errors(vh_ctx* ctx) {
  if (!ctx) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  // a pending surface pass reports into the same word from its own stream
  if (ctx->surf_pending) VH_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->surf_ev, 0));
  VH_CUDA(ctx, cudaMemsetAsync(ctx->f.err, 0, sizeof(unsigned), ctx->stream));
  return VH_OK;
}

vh_status vh_sync(vh_ctx* ctx) {
  unsigned bits = 0;
  vh_status st = vh_error_bits(ctx, &bits);
  if (st != VH_OK) return st;
  if (bits) {
    char buf[160];
    snprintf(buf, sizeof buf,
             "numerical failure during a step (error bits 0x%x: 1 e>1e10, 2 NaN flux, "
             "4 NaN source, 8 inf/NaN shear)",
             bits);
    return fail(ctx, VH_ERR_NUMERIC, buf);
  }
  return VH_OK;
}

vh_status vh_launches_per_step(vh_ctx* ctx, int* n) {
  if (!ctx || !n) return VH_ERR_ARG;
  // update_m, 2 x (faces + update), 2 ghost, the viscous five (prims, the
  // relaxation's list and relaxation, advection, update) and the six of the
  // vorticity, the MLP guess, the clock
  int k = 1 + 2 * (2 + (ctx->g.nz > 1 ? 1 : 0) + 1) + 1 + (ctx->viscous ? 5 : 0) + 1 +
          (ctx->viscous && ctx->vort_on ? 6 : 0) + (ctx->mlp ? 1 : 0) + 1;
  *n = k;
  return VH_OK;
}

vh_status vh_totals(vh_ctx* ctx, double ecrit, double* out) {
  if (!ctx || !out) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_totals: no state uploaded");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::launch_totals(ctx->g, surf_eos(ctx), ctx->f, ctx->tau, ecrit, ctx->grid.etamin, ctx->viscous,
                    ctx->tot_partial, ctx->tot_out, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  double h[vh::kTotals];
  VH_CUDA(ctx, cudaMemcpyAsync(h, ctx->tot_out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const double dx = ctx->g.dx, dy = ctx->g.dy, dz = ctx->g.dz;
  // src/fld.cpp:846-851
  h[0] = h[0] * dx * dy * dz;
  h[1] = h[1] * dx * dy * dz;
  h[2] *= dx * dy * dz;
  h[3] *= dx * dy * dz;
  h[4] = h[4] * dx * dy * dz;
  for (int k = 0; k < vh::kTotals; k++) out[k] = h[k];
  return VH_OK;
}

// block partials of the surface sums (a fixed count keeps them deterministic)
static const int kSurfPartials = 296;

// the buffers every surface or corona call uses, allocated on first use
static vh_status surf_common(vh_ctx* ctx) {
  const vh::Geo& g = ctx->g;
  vh_ctx::Surf& S = ctx->surf;
  vh_status st;
  if (!S.eN) {
    if ((st = dalloc(ctx, &S.eN, g.N)) || (st = dalloc(ctx, &S.eP, g.N)) ||
        (st = dalloc(ctx, &S.blk, std::max(1, vh::surf_count_blocks(g)))) ||
        (st = dalloc(ctx, &S.counters, 2)) ||
        (st = dalloc(ctx, &S.partial, (size_t)(kSurfPartials + 1) * vh::kSurfAcc)))
      return st;
  }
  if (!S.host) {
    static_assert(vh::kSurfAcc == 5, "vh_ctx::Surf::Host::acc");
    VH_CUDA(ctx, cudaHostAlloc((void**)&S.host, sizeof(vh_ctx::Surf::Host), cudaHostAllocDefault));
  }
  return VH_OK;
}

// One pass of outputSurface's element search on the context stream with
// buffers for want_c hypercubes and want_e elements: the nine kernels, the
// beta.dat values when vorticity is on, and the copies of the counts, sums
// and error bits into the pinned host block.  Nothing waits.
static vh_status surf_enqueue(vh_ctx* ctx, double ecrit, size_t want_c, size_t want_e,
                              const vh::Fields& f, double tau, const double* dbeta,
                              cudaStream_t s) {
  const vh::Geo& g = ctx->g;
  vh_ctx::Surf& S = ctx->surf;
  vh_status st;
  if ((st = dgrow(ctx, &S.cubes, &S.cap_cubes, want_c)) ||
      (st = dgrow(ctx, &S.geo, &S.cap_geo, want_c * vh::kSurfMaxElemPerCube * vh::kSurfGeo)) ||
      (st = dgrow(ctx, &S.cnt, &S.cap_cnt, want_c + 1)) ||
      (st = dgrow(ctx, &S.rec, &S.cap_rec, want_e * vh::kSurfRec)) ||
      (st = dgrow(ctx, &S.contrib, &S.cap_contrib, want_e * vh::kSurfAcc)))
    return st;
  if (ctx->vort_on && (st = dgrow(ctx, &ctx->surf_beta, &ctx->cap_beta, want_e * 16))) return st;
  const int cap_c = (int)std::min<size_t>(want_c, INT32_MAX / 16);
  const int cap_e = (int)std::min<size_t>(want_e, INT32_MAX / 32);
  S.pass_cap_c = cap_c;
  S.pass_cap_e = cap_e;
  const double taup = tau - ctx->fluid_dt;
  vh_ctx::Surf::Host& H = *S.host;
  const vh::EosDev SE = surf_eos(ctx);
  vh::launch_surf_energy(g, SE, f, tau, taup, S.eN, S.eP, s);
  vh::launch_surf_count(g, S.eN, S.eP, ecrit, S.blk, S.counters, s);
  vh::launch_surf_compact(g, S.eN, S.eP, ecrit, S.blk, S.cubes, cap_c, s);
  vh::launch_surf_cornelius(g, S.eN, S.eP, ecrit, ctx->fluid_dt, S.cubes, S.counters, cap_c,
                            S.geo, S.cnt, f.err, s);
  vh::launch_surf_elements(g, SE, f, tau, ctx->fluid_dt, ecrit, ctx->grid.xmin,
                           ctx->grid.ymin, ctx->grid.etamin, S.cubes, S.counters, cap_c, cap_e,
                           S.geo, S.cnt, S.rec, S.contrib, S.partial, kSurfPartials, s);
  if (ctx->vort_on)  // beta.dat lines (src/fld.cpp:663-669, 798-831)
    vh::launch_surf_beta(g, dbeta, ctx->grid.etamin, S.cubes, S.counters, cap_c, cap_e, S.geo,
                         S.cnt, ctx->surf_beta, s);
  VH_CUDA(ctx, cudaGetLastError());
  VH_CUDA(ctx, cudaMemcpyAsync(H.cnt, S.counters, sizeof H.cnt, cudaMemcpyDeviceToHost, s));
  VH_CUDA(ctx, cudaMemcpyAsync(H.acc, S.partial + (size_t)kSurfPartials * vh::kSurfAcc,
                               sizeof H.acc, cudaMemcpyDeviceToHost, s));
  VH_CUDA(ctx, cudaMemcpyAsync(&H.bits, ctx->f.err, sizeof H.bits, cudaMemcpyDeviceToHost, s));
  return VH_OK;
}

// The buffers a pass starts with: what earlier calls left, at least 64k
// hypercubes (or all of them) and twice as many elements.
static void surf_want(vh_ctx* ctx, size_t* want_c, size_t* want_e) {
  const long long ninterior = std::max(1LL, vh::surf_ncube(ctx->g));
  *want_c = std::max<size_t>(ctx->surf.cap_cubes, (size_t)std::min(ninterior, 65536LL));
  *want_e = std::max<size_t>(ctx->surf.cap_rec / vh::kSurfRec, 2 * *want_c);
}

// After a pass's copies landed: false when it found more hypercubes or
// elements than its buffers held (then want_c / want_e hold what a pass
// over the same fields needs).
static bool surf_fits(vh_ctx* ctx, size_t* want_c, size_t* want_e) {
  const vh_ctx::Surf& S = ctx->surf;
  const vh_ctx::Surf::Host& H = *S.host;
  if ((size_t)H.cnt[0] <= (size_t)S.pass_cap_c && (size_t)H.cnt[1] <= (size_t)S.pass_cap_e)
    return true;
  *want_c = std::max(*want_c, (size_t)H.cnt[0] + (size_t)H.cnt[0] / 4 + 1);
  // a cube holds at most kSurfMaxElemPerCube elements
  *want_e = std::max(*want_e, (size_t)H.cnt[0] * vh::kSurfMaxElemPerCube);
  return false;
}

// The results of a pass that fit: element count, the carried sums, info.
static vh_status surf_finish(vh_ctx* ctx, vh_surface_info* info) {
  vh_ctx::Surf& S = ctx->surf;
  const vh_ctx::Surf::Host& H = *S.host;
  const int nel = H.cnt[1];
  const unsigned bits = H.bits;
  const double* acc = H.acc;
  S.nel = nel;
  ctx->cells_kind = 1;
  ctx->beta_nel = ctx->vort_on ? nel : 0;
  ctx->EtotSurf += acc[1];
  ctx->nbSurf += acc[2];
  ctx->vEff += acc[3];
  if (info) {
    info->nelements = nel;
    info->nsusp = (long)acc[0];
    info->high_T = (long)acc[4];
    info->EtotSurf = ctx->EtotSurf;
    info->nbSurf = ctx->nbSurf;
    info->vEff = ctx->vEff;
  }
  if (bits & vh::ERR_SURFACE)
    return fail(ctx, VH_ERR_NUMERIC, "vh_surface: a hypercube on which the reference stops");
  return VH_OK;
}

vh_status vh_surface(vh_ctx* ctx, double ecrit, vh_surface_info* info) {
  if (!ctx) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_surface: no state uploaded");
  if (ctx->surf_pending) return fail(ctx, VH_ERR_STATE, "vh_surface: a vh_surface_begin is pending");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh_status st;
  if ((st = surf_common(ctx))) return st;
  // Every stage reads the counts from device memory, so the call waits for
  // the GPU once, at the end.  A call that finds more than the buffers hold
  // grows them and runs again (the fields it reads are unchanged in
  // between, so the result is the same).
  size_t want_c, want_e;
  surf_want(ctx, &want_c, &want_e);
  for (int pass = 0; pass < 2; pass++) {
    if ((st = surf_enqueue(ctx, ecrit, want_c, want_e, ctx->f, ctx->tau, ctx->vort.dbeta,
                           ctx->stream)))
      return st;
    VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (surf_fits(ctx, &want_c, &want_e)) return surf_finish(ctx, info);
  }
  return fail(ctx, VH_ERR_STATE, "vh_surface: element buffers did not grow");
}

vh_status vh_surface_begin(vh_ctx* ctx, double ecrit) {
  if (!ctx) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_surface_begin: no state uploaded");
  if (ctx->surf_pending)
    return fail(ctx, VH_ERR_STATE, "vh_surface_begin: the previous call has not ended");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh_status st;
  if ((st = surf_common(ctx))) return st;
  if (!ctx->surf_ev) VH_CUDA(ctx, cudaEventCreateWithFlags(&ctx->surf_ev, cudaEventDisableTiming));
  if (!ctx->snap_ev) VH_CUDA(ctx, cudaEventCreateWithFlags(&ctx->snap_ev, cudaEventDisableTiming));
  if (!ctx->surf_stream)
    VH_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->surf_stream, cudaStreamNonBlocking));
  // The call's inputs (Q, Qprev, pi, Pi and, with vorticity, dbeta) are
  // copied in stream order (allocated on the first call), and the pass runs
  // on its own stream from that copy, beside the steps the caller queues
  // next; the copy also serves vh_surface_end when the pass overflows.
  vh_ctx::Surf& S = ctx->surf;
  const bool beta = ctx->vort_on;
  const long long N = ctx->g.N;
  const size_t keep = (size_t)(beta ? 41 : 25) * N;
  if ((st = dgrow(ctx, &S.keep, &S.cap_keep, keep))) return st;
  const vh::Fields& f = ctx->f;
  const double* src[5] = {f.Q, f.Qprev, f.pi, f.Pi, ctx->vort.dbeta};
  const int ncomp[5] = {7, 7, 10, 1, 16};
  size_t off = 0;
  for (int k = 0; k < (beta ? 5 : 4); k++) {
    VH_CUDA(ctx, cudaMemcpyAsync(S.keep + off, src[k], sizeof(double) * ncomp[k] * N,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
    off += (size_t)ncomp[k] * N;
  }
  VH_CUDA(ctx, cudaEventRecord(ctx->snap_ev, ctx->stream));
  VH_CUDA(ctx, cudaStreamWaitEvent(ctx->surf_stream, ctx->snap_ev, 0));
  vh::Fields kf = ctx->f;
  kf.Q = S.keep;
  kf.Qprev = S.keep + 7 * N;
  kf.pi = S.keep + 14 * N;
  kf.Pi = S.keep + 24 * N;
  const double* kbeta = beta ? S.keep + 25 * N : nullptr;
  size_t want_c, want_e;
  surf_want(ctx, &want_c, &want_e);
  if ((st = surf_enqueue(ctx, ecrit, want_c, want_e, kf, ctx->tau, kbeta, ctx->surf_stream)))
    return st;
  VH_CUDA(ctx, cudaEventRecord(ctx->surf_ev, ctx->surf_stream));
  S.keep_tau = ctx->tau;
  S.keep_ecrit = ecrit;
  S.keep_beta = beta;
  ctx->surf_pending = true;
  return VH_OK;
}

vh_status vh_surface_end(vh_ctx* ctx, vh_surface_info* info) {
  if (!ctx) return VH_ERR_ARG;
  if (!ctx->surf_pending) return fail(ctx, VH_ERR_STATE, "vh_surface_end: no vh_surface_begin");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  ctx->surf_pending = false;
  VH_CUDA(ctx, cudaEventSynchronize(ctx->surf_ev));
  // what the caller queues next on its stream comes after the pass
  VH_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->surf_ev, 0));
  size_t want_c, want_e;
  surf_want(ctx, &want_c, &want_e);
  if (!surf_fits(ctx, &want_c, &want_e)) {
    // The fields have moved on, but the pass ran from a copy of its inputs:
    // grow the buffers and run it again on that copy, behind whatever the
    // caller queued since, then wait for it.
    vh_ctx::Surf& S = ctx->surf;
    const long long N = ctx->g.N;
    vh::Fields kf = ctx->f;
    kf.Q = S.keep;
    kf.Qprev = S.keep + 7 * N;
    kf.pi = S.keep + 14 * N;
    kf.Pi = S.keep + 24 * N;
    const double* kbeta = S.keep_beta ? S.keep + 25 * N : nullptr;
    vh_status st;
    if ((st = surf_enqueue(ctx, S.keep_ecrit, want_c, want_e, kf, S.keep_tau, kbeta, ctx->stream)))
      return st;
    VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!surf_fits(ctx, &want_c, &want_e))
      return fail(ctx, VH_ERR_STATE, "vh_surface_end: element buffers did not grow");
  }
  return surf_finish(ctx, info);
}

vh_status vh_corona(vh_ctx* ctx, double ecrit, vh_surface_info* info) {
  if (!ctx) return VH_ERR_ARG;
  if (!ctx->uploaded) return fail(ctx, VH_ERR_STATE, "vh_corona: no state uploaded");
  if (ctx->surf_pending) return fail(ctx, VH_ERR_STATE, "vh_corona: a vh_surface_begin is pending");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  const vh::Geo& g = ctx->g;
  vh_ctx::Surf& S = ctx->surf;
  vh_status st;
  if ((st = surf_common(ctx))) return st;
  const long long ninterior = std::max(1LL, vh::surf_ncube(g));
  if (!S.cflag && (st = dalloc(ctx, &S.cflag, (size_t)ninterior))) return st;
  // one element per cube at most: the buffers start at 64k elements and a
  // call that finds more grows them and runs again, as vh_surface does
  size_t want = std::max<size_t>(std::min<size_t>(S.cap_cubes, S.cap_rec / vh::kSurfRec),
                                 (size_t)std::min(ninterior, 65536LL));
  cudaStream_t s = ctx->stream;
  vh_ctx::Surf::Host& H = *S.host;
  for (int pass = 0; pass < 2; pass++) {
    if ((st = dgrow(ctx, &S.cubes, &S.cap_cubes, want)) ||
        (st = dgrow(ctx, &S.rec, &S.cap_rec, want * vh::kSurfRec)) ||
        (st = dgrow(ctx, &S.contrib, &S.cap_contrib, want * vh::kSurfAcc)))
      return st;
    const int cap = (int)std::min<size_t>(want, INT32_MAX / 32);
    vh::launch_surf_energy(g, surf_eos(ctx), ctx->f, ctx->tau, ctx->tau - ctx->fluid_dt, S.eN, S.eP,
                           s);
    vh::launch_corona(g, surf_eos(ctx), ctx->f, ctx->tau, ecrit, ctx->grid.xmin, ctx->grid.ymin,
                      ctx->grid.etamin, S.eN, S.cflag, S.blk, S.counters, S.cubes, cap, S.rec,
                      S.contrib, S.partial, kSurfPartials, s);
    VH_CUDA(ctx, cudaGetLastError());
    VH_CUDA(ctx, cudaMemcpyAsync(H.cnt, S.counters, sizeof(int), cudaMemcpyDeviceToHost, s));
    VH_CUDA(ctx, cudaMemcpyAsync(H.acc, S.partial + (size_t)kSurfPartials * vh::kSurfAcc,
                                 sizeof H.acc, cudaMemcpyDeviceToHost, s));
    VH_CUDA(ctx, cudaStreamSynchronize(s));
    if ((size_t)H.cnt[0] <= (size_t)cap) break;
    if (pass == 1) return fail(ctx, VH_ERR_STATE, "vh_corona: element buffers did not grow");
    want = (size_t)H.cnt[0] + (size_t)H.cnt[0] / 8 + 1;
  }
  const double* acc = H.acc;
  S.nel = H.cnt[0];
  ctx->cells_kind = 2;
  ctx->corona_cells = H.cnt[0];  // Fluid::num_corona_cells, src/fld.cpp:1071
  ctx->beta_nel = 0;             // the corona writes no beta.dat lines
  ctx->EtotSurf += acc[1];
  ctx->nbCorona += acc[2];
  ctx->vEff += acc[3];
  if (info) {
    info->nelements = H.cnt[0];
    info->nsusp = 0;
    info->high_T = (long)acc[4];
    info->EtotSurf = ctx->EtotSurf;
    info->nbSurf = ctx->nbCorona;
    info->vEff = ctx->vEff;
  }
  return VH_OK;
}

vh_status vh_set_slab(vh_ctx* ctx, int own0, int own1, int z_global0, int nz_global) {
  if (!ctx) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_set_slab");
  vh::Geo& g = ctx->g;
  if (own0 < 0 || own1 <= own0 || own1 > g.nz || z_global0 < 0 ||
      (long long)z_global0 + g.nz > nz_global)
    return fail(ctx, VH_ERR_ARG, "vh_set_slab: the owned planes or the slab's place are out of range");
  g.zoff = z_global0;
  g.nzg = nz_global;
  // the whole grid's interior [2, nz_global - 2) in this slab's planes
  const int lo = 2 - z_global0, hi = nz_global - 2 - z_global0;
  g.zc0 = g.zt0 = std::max(own0, lo);
  g.zc1 = g.zt1 = std::max(g.zc0, std::min(own1, hi));
  // a cube's upper corner plane must exist here
  if (g.zc1 > g.nz - 1)
    return fail(ctx, VH_ERR_ARG, "vh_set_slab: an owned cube's upper plane is not in the slab");
  return VH_OK;
}

vh_status vh_surface_cells(vh_ctx* ctx, int* ixyz, long cap, long* n) {
  if (!ctx || (!ixyz && cap > 0)) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_surface_cells");
  if (ctx->cells_kind == 0) return fail(ctx, VH_ERR_STATE, "vh_surface_cells: no freeze-out call yet");
  const vh_ctx::Surf& S = ctx->surf;
  const long long nel = S.nel;
  if (n) *n = (long)nel;
  const long k = (long)std::min<long long>(nel, std::max(0L, cap));
  if (k == 0) return VH_OK;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  const vh::Geo& g = ctx->g;
  const long long niz = g.zc1 - g.zc0, niy = g.ny - 4;
  auto put = [&](long e, int t) {
    ixyz[3 * e + 0] = 2 + (int)(t / (niz * niy));  // cube_cell (vh_surface.cuh)
    ixyz[3 * e + 1] = 2 + (int)((t / niz) % niy);
    ixyz[3 * e + 2] = g.zc0 + (int)(t % niz) + g.zoff;
  };
  if (ctx->cells_kind == 2) {  // a corona element per cube
    std::vector<int> cubes((size_t)k);
    VH_CUDA(ctx, cudaMemcpyAsync(cubes.data(), S.cubes, sizeof(int) * k, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (long e = 0; e < k; e++) put(e, cubes[(size_t)e]);
    return VH_OK;
  }
  const int ncubes = S.host->cnt[0];
  std::vector<int> cubes((size_t)ncubes), off((size_t)ncubes);
  if (ncubes > 0) {
    VH_CUDA(ctx, cudaMemcpyAsync(cubes.data(), S.cubes, sizeof(int) * ncubes,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    VH_CUDA(ctx, cudaMemcpyAsync(off.data(), S.cnt, sizeof(int) * ncubes, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  for (int c = 0; c < ncubes; c++) {
    const long e1 = c + 1 < ncubes ? off[(size_t)c + 1] : (long)nel;
    for (long e = off[(size_t)c]; e < e1 && e < k; e++) put(e, cubes[(size_t)c]);
  }
  return VH_OK;
}

vh_status vh_surface_records(vh_ctx* ctx, double* out, long max, long* n) {
  if (!ctx || (!out && max > 0)) return VH_ERR_ARG;
  if (ctx->surf_pending)
    return fail(ctx, VH_ERR_STATE, "vh_surface_records: a vh_surface_begin is pending");
  const long k = (long)std::min<long long>(ctx->surf.nel, std::max(0L, max));
  if (n) *n = (long)ctx->surf.nel;
  if (k > 0) {
    VH_CUDA(ctx, cudaSetDevice(ctx->device));
    VH_CUDA(ctx, cudaMemcpyAsync(out, ctx->surf.rec, sizeof(double) * vh::kSurfRec * k,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return VH_OK;
}

vh_status vh_surface_device(vh_ctx* ctx, const double** rec, long* n) {
  if (!ctx || !rec || !n) return VH_ERR_ARG;
  *rec = ctx->surf.rec;
  *n = (long)ctx->surf.nel;
  return VH_OK;
}

vh_status vh_surface_write(vh_ctx* ctx, const char* path, int extendFO) {
  if (!ctx || !path) return VH_ERR_ARG;
  const long n = (long)ctx->surf.nel;
  std::vector<double> h((size_t)n * vh::kSurfRec);
  vh_status st = vh_surface_records(ctx, h.data(), n, nullptr);
  if (st != VH_OK) return st;
  std::ofstream out(path, std::ios::app);
  if (!out) return fail(ctx, VH_ERR_ARG, std::string("vh_surface_write: cannot open ") + path);
  // src/fld.cpp:658-797: precision 15, width 24, OUTPI layout
  out.precision(15);
  const int ncol = extendFO ? vh::kSurfRec : vh::kSurfRec - 2;
  for (long i = 0; i < n; i++) {
    const double* r = h.data() + (size_t)i * vh::kSurfRec;
    for (int c = 0; c < ncol; c++) out << std::setw(24) << r[c];
    out << std::endl;
  }
  return out ? VH_OK : fail(ctx, VH_ERR_ARG, "vh_surface_write: write failed");
}

vh_status vh_enable_vorticity(vh_ctx* ctx, int on) {
  if (!ctx) return VH_ERR_ARG;
  VH_NOT_PENDING(ctx, "vh_enable_vorticity");
  const long long N = ctx->g.N;
  if (N > INT32_MAX) return fail(ctx, VH_ERR_ARG, "vh_enable_vorticity: grid too large");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::VortDev& v = ctx->vort;
  if (on && !v.dbeta) {
    vh_status st;
    if ((st = dalloc(ctx, &v.dbeta, (size_t)16 * N)) || (st = dalloc(ctx, &v.TD, (size_t)N)) ||
        (st = dalloc(ctx, &v.val, (size_t)18 * N)) || (st = dalloc(ctx, &v.R, (size_t)2 * N)) ||
        (st = dalloc(ctx, &v.flag, (size_t)N)) || (st = dalloc(ctx, &v.last, (size_t)5 * N)) ||
        (st = dalloc(ctx, &v.agg, (size_t)5 * vh::vort_scan_blocks(N))))
      return st;
    // Cell::enableVorticity, src/cll.h:167-170: dbeta starts at zero
    VH_CUDA(ctx, cudaMemsetAsync(v.dbeta, 0, sizeof(double) * 16 * N, ctx->stream));
  }
  if ((on != 0) != ctx->vort_on) {
    ctx->vort_on = on != 0;
    ctx->version++;  // the captured step changes
  }
  return VH_OK;
}

vh_status vh_vorticity_chain(vh_ctx* ctx, int n) {
  if (!ctx || n < 0 || n > 32) return VH_ERR_ARG;
  ctx->vort.chain = n;
  ctx->version++;  // the captured step holds the value
  return VH_OK;
}

vh_status vh_get_dbeta(vh_ctx* ctx, double* out) {
  if (!ctx || !out) return VH_ERR_ARG;
  if (!ctx->vort.dbeta) return fail(ctx, VH_ERR_STATE, "vh_get_dbeta: vorticity never enabled");
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  VH_CUDA(ctx, cudaMemcpyAsync(out, ctx->vort.dbeta, sizeof(double) * 16 * ctx->g.N,
                               cudaMemcpyDeviceToHost, ctx->stream));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VH_OK;
}

vh_status vh_surface_beta(vh_ctx* ctx, double* out, long max, long* n) {
  if (!ctx || (!out && max > 0)) return VH_ERR_ARG;
  if (ctx->surf_pending)
    return fail(ctx, VH_ERR_STATE, "vh_surface_beta: a vh_surface_begin is pending");
  if (!ctx->vort_on) return fail(ctx, VH_ERR_STATE, "vh_surface_beta: vorticity is off");
  const long k = (long)std::min<long long>(ctx->beta_nel, std::max(0L, max));
  if (n) *n = (long)ctx->beta_nel;
  if (k > 0) {
    if (!ctx->surf_beta || ctx->cap_beta < (size_t)k * 16)
      return fail(ctx, VH_ERR_STATE, "vh_surface_beta: no vh_surface call with vorticity on");
    VH_CUDA(ctx, cudaSetDevice(ctx->device));
    VH_CUDA(ctx, cudaMemcpyAsync(out, ctx->surf_beta, sizeof(double) * 16 * k,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return VH_OK;
}

vh_status vh_surface_write_beta(vh_ctx* ctx, const char* path, int header) {
  if (!ctx || !path) return VH_ERR_ARG;
  std::ofstream out(path, std::ios::app);
  if (!out) return fail(ctx, VH_ERR_ARG, std::string("vh_surface_write_beta: cannot open ") + path);
  if (header) {
    // Fluid::printDbetaHeader, src/fld.cpp:174-188 (the reference throws
    // before outputCorona has counted the corona cells)
    if (ctx->corona_cells < 0)
      return fail(ctx, VH_ERR_STATE, "vh_surface_write_beta: no vh_corona call yet (header)");
    out << "# The derivatives of \u03b2 are given in Cartesian coordinates and include a "
           "factor of 1/2, such that \u2202\u2098\u03b2\u2099=1/2 * "
           "\u2202\u2098(u\u2099/T)"
        << std::endl;
    out << "# Number of corona cells: " << ctx->corona_cells << std::endl;
    out << "#  \u03c4  x  y  \u03b7  d\u03a3[0]  d\u03a3[1]  d\u03a3[2]  d\u03a3[3]  "
        << "u[0]  u[1]  u[2]  u[3]  T  \u03bcB  \u03bcQ  \u03bcS  "
        << "\u2202\u2080\u03b2\u2080  \u2202\u2080\u03b2\u2081  \u2202\u2080\u03b2\u2082  "
           "\u2202\u2080\u03b2\u2083  \u2202\u2081\u03b2\u2080  \u2202\u2081\u03b2\u2081  "
           "\u2202\u2081\u03b2\u2082  \u2202\u2081\u03b2\u2083  "
        << "\u2202\u2082\u03b2\u2080  \u2202\u2082\u03b2\u2081  \u2202\u2082\u03b2\u2082  "
           "\u2202\u2082\u03b2\u2083  \u2202\u2083\u03b2\u2080  \u2202\u2083\u03b2\u2081  "
           "\u2202\u2083\u03b2\u2082  \u2202\u2083\u03b2\u2083  \u03f5"
        << std::endl;
  }
  const long n = (long)ctx->beta_nel;
  if (n > 0) {
    std::vector<double> rec((size_t)n * vh::kSurfRec), beta((size_t)n * 16);
    vh_status st = vh_surface_records(ctx, rec.data(), n, nullptr);
    if (st == VH_OK) st = vh_surface_beta(ctx, beta.data(), n, nullptr);
    if (st != VH_OK) return st;
    // src/fld.cpp:663-669, 741-745, 826-830: precision 15, width 24
    out.precision(15);
    for (long i = 0; i < n; i++) {
      const double* r = rec.data() + (size_t)i * vh::kSurfRec;
      for (int c = 0; c < 16; c++) out << std::setw(24) << r[c];
      for (int c = 0; c < 16; c++) out << std::setw(24) << beta[(size_t)i * 16 + c];
      out << std::setw(24) << r[27] << std::endl;
    }
  }
  return out ? VH_OK : fail(ctx, VH_ERR_ARG, "vh_surface_write_beta: write failed");
}

vh_status vh_cornelius4d(const double* cubes, long n, const double* dx, double e0, int device,
                         int* counts, double* cent, double* norm) {
  if (n < 0 || n > (1L << 24) || (n > 0 && (!cubes || !dx || !counts || !cent || !norm)))
    return fail(nullptr, VH_ERR_ARG, "vh_cornelius4d: bad arguments");
  if (n == 0) return VH_OK;
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
  double *dc = nullptr, *dg = nullptr;
  int* dn = nullptr;
  const size_t G = (size_t)vh::kSurfMaxElemPerCube * vh::kSurfGeo;
  std::vector<double> hg((size_t)n * G);
  if ((e = cudaMalloc(&dc, sizeof(double) * 16 * n)) == cudaSuccess &&
      (e = cudaMalloc(&dg, sizeof(double) * G * n)) == cudaSuccess &&
      (e = cudaMalloc(&dn, sizeof(int) * n)) == cudaSuccess &&
      (e = cudaMemcpy(dc, cubes, sizeof(double) * 16 * n, cudaMemcpyHostToDevice)) == cudaSuccess) {
    vh::launch_cornelius_batch(dc, (int)n, dx, e0, dn, dg, 0);
    if ((e = cudaGetLastError()) == cudaSuccess &&
        (e = cudaMemcpy(counts, dn, sizeof(int) * n, cudaMemcpyDeviceToHost)) == cudaSuccess)
      e = cudaMemcpy(hg.data(), dg, sizeof(double) * G * n, cudaMemcpyDeviceToHost);
  }
  cudaFree(dc);
  cudaFree(dg);
  cudaFree(dn);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "vh_cornelius4d");
  for (long k = 0; k < n; k++)
    for (int el = 0; el < vh::kSurfMaxElemPerCube; el++)
      for (int d = 0; d < 4; d++) {
        cent[(k * vh::kSurfMaxElemPerCube + el) * 4 + d] = hg[k * G + el * vh::kSurfGeo + d];
        norm[(k * vh::kSurfMaxElemPerCube + el) * 4 + d] = hg[k * G + el * vh::kSurfGeo + 4 + d];
      }
  return VH_OK;
}

vh_status vh_timer_start(vh_ctx* ctx) {
  if (!ctx) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->t0) VH_CUDA(ctx, cudaEventCreate(&ctx->t0));
  if (!ctx->t1) VH_CUDA(ctx, cudaEventCreate(&ctx->t1));
  VH_CUDA(ctx, cudaEventRecord(ctx->t0, ctx->stream));
  return VH_OK;
}

vh_status vh_timer_stop(vh_ctx* ctx, double* ms) {
  if (!ctx || !ms || !ctx->t0) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  VH_CUDA(ctx, cudaEventRecord(ctx->t1, ctx->stream));
  VH_CUDA(ctx, cudaEventSynchronize(ctx->t1));
  float f = 0.f;
  VH_CUDA(ctx, cudaEventElapsedTime(&f, ctx->t0, ctx->t1));
  *ms = f;
  return VH_OK;
}

int vh_profile_kinds(void) { return vh::KK_COUNT; }

vh_status vh_profile_enable(vh_ctx* ctx, int on) {
  if (!ctx) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->prof = on != 0;
  ctx->segs.clear();
  ctx->evused = 0;
  return VH_OK;
}

vh_status vh_profile_read(vh_ctx* ctx, int kind, const char** name, long* launches,
                          double* total_ms) {
  if (!ctx || kind < 0 || kind >= vh::KK_COUNT) return VH_ERR_ARG;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  VH_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  long n = 0;
  double tot = 0.;
  for (const auto& sg : ctx->segs) {
    if (sg.kind != kind) continue;
    float f = 0.f;
    VH_CUDA(ctx, cudaEventElapsedTime(&f, ctx->evpool[sg.ev0], ctx->evpool[sg.ev1]));
    tot += f;
    n++;
  }
  if (name) *name = vh::kKernelNames[kind];
  if (launches) *launches = n;
  if (total_ms) *total_ms = tot;
  return VH_OK;
}

vh_status vh_alloc_pinned(size_t bytes, void** p) {
  if (!p) return VH_ERR_ARG;
  cudaError_t e = cudaHostAlloc(p, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) return fail(nullptr, VH_ERR_CUDA, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
  return VH_OK;
}

vh_status vh_free_pinned(void* p) {
  if (p) cudaFreeHost(p);
  return VH_OK;
}

vh_status vh_transform_pv(vh_ctx* ctx, const double* Q_dev, long n, double* prim_dev) {
  if (!ctx || !Q_dev || !prim_dev || n < 0) return VH_ERR_ARG;
  if (n == 0) return VH_OK;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::launch_transform_pv(ctx->eos, Q_dev, (long long)n, prim_dev, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  return VH_OK;
}

vh_status vh_transport_eval(vh_ctx* ctx, const double* in_dev, long n, double* out_dev) {
  if (!ctx || !in_dev || !out_dev || n < 0) return VH_ERR_ARG;
  if (n == 0) return VH_OK;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::launch_transport(ctx->tr, in_dev, (long long)n, out_dev, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  return VH_OK;
}

vh_status vh_eos_eval(vh_ctx* ctx, const double* e_dev, const double* nb_dev, long n,
                      double* out_dev) {
  if (!ctx || !e_dev || !nb_dev || !out_dev || n < 0) return VH_ERR_ARG;
  if (n == 0) return VH_OK;
  VH_CUDA(ctx, cudaSetDevice(ctx->device));
  vh::launch_eos_eval(ctx->eos, e_dev, nb_dev, (long long)n, out_dev, ctx->stream);
  VH_CUDA(ctx, cudaGetLastError());
  return VH_OK;
}

}  // extern "C"
