// vh_ctx.cuh -- the context behind the C ABI's opaque vh_ctx (one grid on
// one GPU), shared by the ABI implementation files.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/vhlle_b200.h"
#include "vh_mlp.cuh"
#include "vh_step.cuh"

struct vh_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  vh::Geo g{};
  vh::EosDev eos{};
  // Fluid's eosH (vh_set_surface_eos): the EoS of the surface, the corona
  // and the totals when has_eosH; else the hydro EoS
  vh::EosDev eosH{};
  bool has_eosH = false;
  vh::TrDev tr{};
  vh::Fields f{};
  double tau = 0., dt = 0.;
  bool viscous = false;
  bool uploaded = false;
  int launches = 0;
  vh_grid grid{};
  double* tot_partial = nullptr;  // [blocks][16] block sums of the totals
  double* tot_out = nullptr;      // [16]
  double* resize_tmp = nullptr;   // [10][N] staging of the resize gather
  double* clk = nullptr;          // [2] device clock (tau, dt) the step kernels read
  unsigned long long* c2p_stats = nullptr;  // [2] con2prim calls, iterations
  int version = 0;  // bumped by every change a captured step bakes in
  // vh_step replays one captured step per fill-fraction buffer order
  // (f.m == m_first or not) while `version` is unchanged: one graph launch
  // per step instead of ~20 kernel launches (captured on a private stream,
  // launched on `stream`); steps with per-kernel profiling launch directly
  cudaStream_t cap_stream = nullptr;
  // vh_step_host: the step with its host copies, per fill-fraction buffer
  // order, for one buffer set (host_key) at the version it was captured at
  cudaGraphExec_t host_exec[2] = {nullptr, nullptr};
  int host_version[2] = {-1, -1};
  std::vector<const void*> host_key[2];
  cudaStream_t copy_up = nullptr, copy_down = nullptr;
  cudaEvent_t host_ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t step_exec[2] = {nullptr, nullptr};
  int step_version[2] = {-1, -1};
  int step_launches[2] = {0, 0};
  bool step_graphs = true;  // false after a capture was refused (e.g. inside
                            // a caller's own global-mode capture)
  double* m_first = nullptr;
  vh_mlp* mlp = nullptr;           // learned con2prim start point (not owned)
  float* vguess = nullptr;         // [N] per-cell start points of the step
  unsigned long long* ucount = nullptr;
  // the Fluid's construction-time step: the time side of the freeze-out
  // hypercubes (src/fld.cpp:106-108); set at creation, doubled by the resize
  double fluid_dt = 0.;
  // surface sums: EtotSurf and vEff are Fluid members (reset by the resize's
  // new Fluid), nbSurf is a function static in the reference (never reset)
  double EtotSurf = 0., vEff = 0., nbSurf = 0.;
  double nbCorona = 0.;  // outputCorona's own function static (src/fld.cpp:877)
  // vorticity (Hydro::enableVorticity): buffers allocated on the first enable
  bool vort_on = false;
  vh::VortDev vort{};
  double* surf_beta = nullptr;  // [cap][16] beta.dat values of the last vh_surface
  size_t cap_beta = 0;
  long long beta_nel = 0;       // its element count (0 after vh_corona)
  int cells_kind = 0;           // the last freeze-out call: 1 vh_surface, 2 vh_corona
  long long corona_cells = -1;  // elements of the last vh_corona (the beta.dat header)
  // vh_surface_begin / vh_surface_end: one call in flight, its completion event
  bool surf_pending = false;
  cudaEvent_t surf_ev = nullptr;
  // a pipelined surface call runs on its own stream from a snapshot of its
  // inputs, beside the steps that follow it
  cudaStream_t surf_stream = nullptr;
  cudaEvent_t snap_ev = nullptr;
  struct Surf {
    double *eN = nullptr, *eP = nullptr, *geo = nullptr, *rec = nullptr, *contrib = nullptr,
           *partial = nullptr;
    int *blk = nullptr, *cubes = nullptr, *cnt = nullptr, *counters = nullptr;
    unsigned char* cflag = nullptr;  // [interior cubes] corona flags
    size_t cap_cubes = 0, cap_geo = 0, cap_cnt = 0, cap_rec = 0, cap_contrib = 0;
    int pass_cap_c = 0, pass_cap_e = 0;  // the buffers the last pass ran with
    long long nel = 0;
    // a pipelined call's copy of Q, Qprev, pi, Pi (and dbeta with vorticity
    // on), written on the device only when its pass overflowed, and the
    // call's tau and e_crit: vh_surface_end runs the pass again from them
    double* keep = nullptr;
    size_t cap_keep = 0;
    double keep_tau = 0., keep_ecrit = 0.;
    bool keep_beta = false;
    // pinned landing place of a call's counts, sums and error bits
    struct Host {
      int cnt[2];
      unsigned bits;
      double acc[5];
    }* host = nullptr;
  } surf;
  std::string err;
  std::vector<void*> allocs;
  // timers and per-kernel profiling
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  bool prof = false;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
  struct Seg {
    int kind;
    size_t ev0, ev1;
  };
  std::vector<Seg> segs;
};
