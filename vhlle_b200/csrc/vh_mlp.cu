// vh_mlp.cu -- the learned start point for the con2prim root find.
//
// A 4 -> 64 -> 64 -> 3 MLP (SiLU, BF16 weights and activations, FP32
// accumulation) maps a cell's conserved state to (e/T^00, |v|, nb/T^00).
// Its |v| is the start point of every con2prim of that cell in the step; the
// FP64 safeguarded Newton / bisection of transformPV (src/rmn.cpp:28-139)
// still finishes every solve to the context's tolerance, so the network only
// changes the iteration count.
//
//   inference  k_mlp_guess / k_mlp_forward: one warp per 16 cells, the three
//              layers as BF16 mma.sync m16n8k16 tiles (the 64-wide layers
//              are far too small for a CTA-level tcgen05 pipeline to pay:
//              this runs once per cell per step, ~45 MMAs per 16 cells);
//              the FP32 accumulators of one layer become the next layer's A
//              fragments in registers.
//   training   k_mlp_grad (forward + backward for 128 samples per block, the
//              weight gradients as block-level FP32 GEMMs in shared memory,
//              one global atomic per parameter per block), k_mlp_adam.
//   data       k_mlp_samples: features of every cell's Q/tau with labels
//              from transformPV at the tight tolerance.
//
// Features x = (0.1 ln T^00, min(|T^0i|/T^00, 1.5), J^0/T^00, [|T^0i| > T^00]),
// T^0mu = Q/tau.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "vh_mlp.cuh"
#include "vh_physics.cuh"

namespace vh {

// FP32 master parameter offsets
constexpr int kW1 = 0, kB1 = 256, kW2 = 320, kB2 = 4416, kW3 = 4480, kB3 = 4672;
static_assert(kB3 + 3 == kMlpParams, "parameter layout");

// packed inference weights (32-bit words of two bf16, rows padded so that
// the B-fragment loads of a warp hit 32 distinct banks)
constexpr int kP1Stride = 12, kP2Stride = 36, kP3Stride = 36;
constexpr int kP1 = 0, kP2 = kP1 + 64 * kP1Stride, kP3 = kP2 + 64 * kP2Stride,
              kPWords = kP3 + 8 * kP3Stride;
constexpr int kPBias = kPWords;  // then b1[64], b2[64], b3[8] as floats
constexpr int kPackWords = kPBias + 136;

__device__ __forceinline__ float bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
// SiLU for inference: z sigmoid(z) = z (1 + tanh(z / 2)) / 2 with the
// hardware tanh (one transcendental-unit operation instead of an exp and a
// reciprocal; relative error ~2^-11, below the BF16 rounding of the
// activations that follows).  The exp and the divide of silu() kept the
// transcendental unit of the inference kernel 58 % busy.
__device__ __forceinline__ float tanh_hw(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float silu_fast(float z) { return 0.5f * z * (1.f + tanh_hw(0.5f * z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ bool mlp_features(const double q[7], float x[4]) {
  const double QT = q[T_];
  if (!(QT > 0.)) return false;
  const double M = sqrt(q[X_] * q[X_] + q[Y_] * q[Y_] + q[Z_] * q[Z_]);
  if (!(M > 0.)) return false;
  x[0] = 0.1f * (float)log(QT);
  x[1] = (float)fmin(M / QT, 1.5);
  x[2] = (float)(q[NB_] / QT);
  x[3] = M > QT ? 1.f : 0.f;
  return true;
}

// ------------------------------------------------------------ inference
__global__ void k_mlp_pack(const float* __restrict__ P, uint32_t* __restrict__ out) {
  for (int w = threadIdx.x + blockIdx.x * blockDim.x; w < kPackWords;
       w += blockDim.x * gridDim.x) {
    uint32_t v = 0;
    if (w < kP2) {
      const int n = w / kP1Stride, c = w % kP1Stride, k = 2 * c;
      const float a = k < 4 ? P[kW1 + n * 4 + k] : 0.f, b = k + 1 < 4 ? P[kW1 + n * 4 + k + 1] : 0.f;
      v = c < 8 ? pack2(a, b) : 0u;
    } else if (w < kP3) {
      const int r = w - kP2, n = r / kP2Stride, c = r % kP2Stride, k = 2 * c;
      v = c < 32 ? pack2(P[kW2 + n * 64 + k], P[kW2 + n * 64 + k + 1]) : 0u;
    } else if (w < kPWords) {
      const int r = w - kP3, n = r / kP3Stride, c = r % kP3Stride, k = 2 * c;
      v = (c < 32 && n < 3) ? pack2(P[kW3 + n * 64 + k], P[kW3 + n * 64 + k + 1]) : 0u;
    } else {
      const int b = w - kPBias;
      const float f = b < 64 ? P[kB1 + b] : (b < 128 ? P[kB2 + b - 64] : (b - 128 < 3 ? P[kB3 + b - 128] : 0.f));
      v = __float_as_uint(f);
    }
    out[w] = v;
  }
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One warp evaluates 16 rows (cells).  feat: this warp's [16][4] features in
// shared memory (rows without a state are zero).  Returns, for lanes with
// (lane & 3) == 0, the outputs of rows g = lane >> 2 and g + 8 in out0/out1
// (three values each).
__device__ __forceinline__ void mlp_warp(const uint32_t* __restrict__ W, const float (*feat)[4],
                                         float out0[3], float out1[3]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const float* bias = reinterpret_cast<const float*>(W + kPBias);
  // layer 1: A = features (k 0..3 of 16)
  uint32_t a[4];
  a[0] = t < 2 ? pack2(feat[g][2 * t], feat[g][2 * t + 1]) : 0u;
  a[1] = t < 2 ? pack2(feat[g + 8][2 * t], feat[g + 8][2 * t + 1]) : 0u;
  a[2] = 0u;
  a[3] = 0u;
  uint32_t h[4][4];  // next layer's A fragments, 4 k-tiles
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float c[4];
    c[0] = c[2] = bias[8 * j + 2 * t];
    c[1] = c[3] = bias[8 * j + 2 * t + 1];
    const uint32_t* wr = W + kP1 + (8 * j + g) * kP1Stride;
    mma_bf16(c, a, wr[t], wr[t + 4]);
    const uint32_t lo = pack2(silu_fast(c[0]), silu_fast(c[1])), hi = pack2(silu_fast(c[2]), silu_fast(c[3]));
    if (j & 1) {
      h[j >> 1][2] = lo;
      h[j >> 1][3] = hi;
    } else {
      h[j >> 1][0] = lo;
      h[j >> 1][1] = hi;
    }
  }
  // layer 2
  uint32_t h2[4][4];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float c[4];
    c[0] = c[2] = bias[64 + 8 * j + 2 * t];
    c[1] = c[3] = bias[64 + 8 * j + 2 * t + 1];
    const uint32_t* wr = W + kP2 + (8 * j + g) * kP2Stride;
#pragma unroll
    for (int kt = 0; kt < 4; kt++) mma_bf16(c, h[kt], wr[8 * kt + t], wr[8 * kt + t + 4]);
    const uint32_t lo = pack2(silu_fast(c[0]), silu_fast(c[1])), hi = pack2(silu_fast(c[2]), silu_fast(c[3]));
    if (j & 1) {
      h2[j >> 1][2] = lo;
      h2[j >> 1][3] = hi;
    } else {
      h2[j >> 1][0] = lo;
      h2[j >> 1][1] = hi;
    }
  }
  // layer 3 (3 outputs in an 8-wide tile)
  float c[4];
  c[0] = c[2] = bias[128 + 2 * t];
  c[1] = c[3] = bias[128 + 2 * t + 1];
  const uint32_t* wr = W + kP3 + g * kP3Stride;
#pragma unroll
  for (int kt = 0; kt < 4; kt++) mma_bf16(c, h2[kt], wr[8 * kt + t], wr[8 * kt + t + 4]);
  // columns 2t, 2t+1 of rows g and g+8; gather the three outputs to lane t=0
  const float c2a = __shfl_down_sync(0xffffffffu, c[0], 1);
  const float c2b = __shfl_down_sync(0xffffffffu, c[2], 1);
  out0[0] = c[0];
  out0[1] = c[1];
  out0[2] = c2a;
  out1[0] = c[2];
  out1[1] = c[3];
  out1[2] = c2b;
}

constexpr int kMlpBlock = 128;  // 4 warps, 64 rows per block pass

__global__ void __launch_bounds__(kMlpBlock) k_mlp_forward(const uint32_t* __restrict__ Wg,
                                                           const float* __restrict__ X, long long n,
                                                           float* __restrict__ Y) {
  __shared__ uint32_t W[kPackWords];
  __shared__ float feat[kMlpBlock / 32][16][4];
  for (int w = threadIdx.x; w < kPackWords; w += kMlpBlock) W[w] = Wg[w];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntile = (n + 15) / 16;
  for (long long tile = (long long)blockIdx.x * (kMlpBlock / 32) + warp; tile < ntile;
       tile += (long long)gridDim.x * (kMlpBlock / 32)) {
    if (lane < 16) {
      const long long r = tile * 16 + lane;
#pragma unroll
      for (int k = 0; k < 4; k++) feat[warp][lane][k] = r < n ? X[r * 4 + k] : 0.f;
    }
    __syncwarp();
    float o0[3], o1[3];
    mlp_warp(W, feat[warp], o0, o1);
    if ((lane & 3) == 0) {
      const long long r0 = tile * 16 + (lane >> 2), r1 = r0 + 8;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        if (r0 < n) Y[r0 * 3 + k] = o0[k];
        if (r1 < n) Y[r1 * 3 + k] = o1[k];
      }
    }
    __syncwarp();
  }
}

// The per-cell start point of a step: |v| of the network for Q/tau, clamped
// into (0, 1); -1 (no guess) where the state has no root to find.
__global__ void __launch_bounds__(kMlpBlock) k_mlp_guess(const uint32_t* __restrict__ Wg,
                                                         const double* __restrict__ Q, long long N,
                                                         const double* __restrict__ clk,
                                                         float* __restrict__ vg) {
  const double tau = clk[0];
  __shared__ uint32_t W[kPackWords];
  __shared__ float feat[kMlpBlock / 32][16][4];
  __shared__ unsigned char okv[kMlpBlock / 32][16];
  for (int w = threadIdx.x; w < kPackWords; w += kMlpBlock) W[w] = Wg[w];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntile = (N + 15) / 16;
  for (long long tile = (long long)blockIdx.x * (kMlpBlock / 32) + warp; tile < ntile;
       tile += (long long)gridDim.x * (kMlpBlock / 32)) {
    if (lane < 16) {
      const long long i = tile * 16 + lane;
      float x[4] = {0.f, 0.f, 0.f, 0.f};
      bool ok = false;
      if (i < N) {
        double q[7];
        // the features are ratios and a float log: Q times RN(1/tau) is
        // as good as Q / tau for them, and takes no divide per component
        const double rtau = 1.0 / tau;
#pragma unroll
        for (int k = 0; k < 7; k++) q[k] = Q[k * N + i] * rtau;
        ok = mlp_features(q, x);
      }
      okv[warp][lane] = ok;
#pragma unroll
      for (int k = 0; k < 4; k++) feat[warp][lane][k] = ok ? x[k] : 0.f;
    }
    __syncwarp();
    float o0[3], o1[3];
    mlp_warp(W, feat[warp], o0, o1);
    if ((lane & 3) == 0) {
      const int g = lane >> 2;
      const long long r0 = tile * 16 + g, r1 = r0 + 8;
      if (r0 < N) vg[r0] = okv[warp][g] ? fminf(fmaxf(o0[1], 1e-4f), 1.f - 1e-4f) : -1.f;
      if (r1 < N) vg[r1] = okv[warp][g + 8] ? fminf(fmaxf(o1[1], 1e-4f), 1.f - 1e-4f) : -1.f;
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------- samples
__global__ void k_mlp_samples(EosDev E, const double* __restrict__ Q, long long N, double tau,
                              float* __restrict__ X, float* __restrict__ Y, long long cap,
                              unsigned long long* __restrict__ count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double q[7];
#pragma unroll
  for (int k = 0; k < 7; k++) q[k] = Q[k * N + i] / tau;
  float x[4];
  if (!mlp_features(q, x)) return;
  const double QT = q[T_];
  Prim P;
  transform_pv(E, q, P);
  const unsigned long long s = atomicAdd(count, 1ull);
  if ((long long)s >= cap) return;
#pragma unroll
  for (int k = 0; k < 4; k++) X[s * 4 + k] = x[k];
  Y[s * 3 + 0] = (float)(P.e / QT);
  Y[s * 3 + 1] = (float)sqrt(P.vx * P.vx + P.vy * P.vy + P.vz * P.vz);
  Y[s * 3 + 2] = (float)(P.nb / QT);
}

// ------------------------------------------------------------- training
constexpr int kTB = 128;  // samples per block
constexpr int kPad = 65;
__constant__ float kLossW[3] = {1.f, 4.f, 1.f};

// Forward + backward for the samples idx(b) = (off + b * stride) mod n,
// b in [b0, b0 + cnt): weight gradients summed into G (global, atomics),
// the summed weighted squared error into loss.  scale = 1 / batch size.
__global__ void __launch_bounds__(kTB) k_mlp_grad(const float* __restrict__ P,
                                                  const float* __restrict__ X,
                                                  const float* __restrict__ Y, long long n,
                                                  long long off, long long stride, long long cnt,
                                                  float scale, float* __restrict__ G,
                                                  float* __restrict__ loss) {
  extern __shared__ float sm[];
  float* Wr = sm;                 // bf16-rounded weights, FP32 biases [kMlpParams]
  float* h1 = Wr + kMlpParams;    // [kTB][kPad]
  float* h2 = h1 + kTB * kPad;
  float* d2 = h2 + kTB * kPad;    // dL/dz2
  float* d1 = d2 + kTB * kPad;    // dL/dz1
  float* xs = d1 + kTB * kPad;    // [kTB][4]
  float* dy = xs + kTB * 4;       // [kTB][4]
  float* red = dy + kTB * 4;      // [kTB]
  const int t = threadIdx.x;
  for (int p = t; p < kMlpParams; p += kTB) {
    const bool bias = (p >= kB1 && p < kW2) || (p >= kB2 && p < kW3) || p >= kB3;
    Wr[p] = bias ? P[p] : bf16r(P[p]);
  }
  __syncthreads();
  const long long b = (long long)blockIdx.x * kTB + t;
  const bool act = b < cnt;
  float z1[64], z2[64];
  float l = 0.f;
  if (act) {
    const long long r = (off + b * stride) % n;
    float x[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      x[k] = bf16r(X[r * 4 + k]);
      xs[t * 4 + k] = x[k];
    }
#pragma unroll 4
    for (int o = 0; o < 64; o++) {
      float a = Wr[kB1 + o];
#pragma unroll
      for (int k = 0; k < 4; k++) a += Wr[kW1 + o * 4 + k] * x[k];
      z1[o] = a;
      h1[t * kPad + o] = bf16r(silu(a));
    }
#pragma unroll 2
    for (int o = 0; o < 64; o++) {
      float a = Wr[kB2 + o];
      for (int k = 0; k < 64; k++) a += Wr[kW2 + o * 64 + k] * h1[t * kPad + k];
      z2[o] = a;
      h2[t * kPad + o] = bf16r(silu(a));
    }
    float dyl[3];
#pragma unroll
    for (int o = 0; o < 3; o++) {
      float a = Wr[kB3 + o];
      for (int k = 0; k < 64; k++) a += Wr[kW3 + o * 64 + k] * h2[t * kPad + k];
      const float e = a - Y[r * 3 + o];
      l += kLossW[o] * e * e;
      dyl[o] = 2.f * kLossW[o] * e * scale;
      dy[t * 4 + o] = dyl[o];
    }
    for (int k = 0; k < 64; k++) {
      const float dh = Wr[kW3 + k] * dyl[0] + Wr[kW3 + 64 + k] * dyl[1] + Wr[kW3 + 128 + k] * dyl[2];
      d2[t * kPad + k] = dh * silu_grad(z2[k]);
    }
    for (int k = 0; k < 64; k++) {
      float dh = 0.f;
      for (int o = 0; o < 64; o++) dh += Wr[kW2 + o * 64 + k] * d2[t * kPad + o];
      d1[t * kPad + k] = dh * silu_grad(z1[k]);
    }
  } else {
    for (int k = 0; k < 64; k++) h1[t * kPad + k] = h2[t * kPad + k] = d2[t * kPad + k] = d1[t * kPad + k] = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) xs[t * 4 + k] = dy[t * 4 + k] = 0.f;
  }
  red[t] = l;
  __syncthreads();
  // weight gradients: sums over the block's samples
  for (int p = t; p < kMlpParams; p += kTB) {
    float a = 0.f;
    if (p < kB1) {
      const int o = p / 4, k = p % 4;
      for (int s = 0; s < kTB; s++) a += d1[s * kPad + o] * xs[s * 4 + k];
    } else if (p < kW2) {
      const int o = p - kB1;
      for (int s = 0; s < kTB; s++) a += d1[s * kPad + o];
    } else if (p < kB2) {
      const int o = (p - kW2) / 64, k = (p - kW2) % 64;
      for (int s = 0; s < kTB; s++) a += d2[s * kPad + o] * h1[s * kPad + k];
    } else if (p < kW3) {
      const int o = p - kB2;
      for (int s = 0; s < kTB; s++) a += d2[s * kPad + o];
    } else if (p < kB3) {
      const int o = (p - kW3) / 64, k = (p - kW3) % 64;
      for (int s = 0; s < kTB; s++) a += dy[s * 4 + o] * h2[s * kPad + k];
    } else {
      const int o = p - kB3;
      for (int s = 0; s < kTB; s++) a += dy[s * 4 + o];
    }
    atomicAdd(&G[p], a);
  }
  if (t == 0) {
    float s = 0.f;
    for (int k = 0; k < kTB; k++) s += red[k];
    atomicAdd(loss, s);
  }
}

__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ G,
                           float* __restrict__ m, float* __restrict__ v, float lr, float b1c,
                           float b2c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float g = G[i];
  const float mi = 0.9f * m[i] + 0.1f * g, vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi / b1c) / (sqrtf(vi / b2c) + 1e-8f);
}

size_t mlp_grad_smem() { return sizeof(float) * (kMlpParams + 4 * kTB * kPad + 8 * kTB + kTB); }

// ----------------------------------------------------------- launchers
void launch_mlp_pack(const float* P, uint32_t* packed, cudaStream_t s) {
  k_mlp_pack<<<(kPackWords + 255) / 256, 256, 0, s>>>(P, packed);
}
int mlp_pack_words() { return kPackWords; }

void launch_mlp_forward(const uint32_t* W, const float* X, long long n, float* Y, cudaStream_t s) {
  const long long tiles = (n + 15) / 16;
  long long blocks = (tiles + 3) / 4;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks > 0) k_mlp_forward<<<(unsigned)blocks, kMlpBlock, 0, s>>>(W, X, n, Y);
}

void launch_mlp_guess(const uint32_t* W, const double* Q, long long N, const double* clk, float* vg,
                      cudaStream_t s) {
  const long long tiles = (N + 15) / 16;
  long long blocks = (tiles + 3) / 4;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks > 0) k_mlp_guess<<<(unsigned)blocks, kMlpBlock, 0, s>>>(W, Q, N, clk, vg);
}

void launch_mlp_samples(const EosDev& E, const double* Q, long long N, double tau, float* X,
                        float* Y, long long cap, unsigned long long* count, cudaStream_t s) {
  if (N > 0) k_mlp_samples<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(E, Q, N, tau, X, Y, cap, count);
}

cudaError_t launch_mlp_grad(const float* P, const float* X, const float* Y, long long n,
                            long long off, long long stride, long long cnt, float* G, float* loss,
                            cudaStream_t s) {
  static bool attr = false;
  const size_t smem = mlp_grad_smem();
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const long long blocks = (cnt + kTB - 1) / kTB;
  if (blocks > 0)
    k_mlp_grad<<<(unsigned)blocks, kTB, smem, s>>>(P, X, Y, n, off, stride, cnt, 1.f / (float)cnt,
                                                   G, loss);
  return cudaGetLastError();
}

void launch_mlp_adam(float* P, const float* G, float* m, float* v, float lr, float b1c, float b2c,
                     cudaStream_t s) {
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(P, G, m, v, lr, b1c, b2c);
}

}  // namespace vh

// ================================================================ C ABI
#include <algorithm>
#include <random>

#include "../../include/vhlle_b200.h"

namespace {
thread_local std::string g_mlp_error;

vh_status mlp_fail(vh_status st, const std::string& m) {
  g_mlp_error = m;
  return st;
}
vh_status mlp_cuda(cudaError_t e, const char* where) {
  return mlp_fail(VH_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define MLP_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return mlp_cuda(e_, #call);   \
  } while (0)

long long gcdll(long long a, long long b) {
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}
}  // namespace

extern "C" {

const char* vh_mlp_last_error(void) { return g_mlp_error.c_str(); }

vh_status vh_mlp_destroy(vh_mlp* m) {
  if (!m) return VH_OK;
  cudaSetDevice(m->device);
  cudaFree(m->P);
  cudaFree(m->G);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->loss);
  cudaFree(m->packed);
  delete m;
  return VH_OK;
}

vh_status vh_mlp_set_params(vh_mlp* m, const float* host) {
  if (!m || !host) return mlp_fail(VH_ERR_ARG, "vh_mlp_set_params: NULL argument");
  MLP_CUDA(cudaSetDevice(m->device));
  MLP_CUDA(cudaMemcpy(m->P, host, sizeof(float) * vh::kMlpParams, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemset(m->m, 0, sizeof(float) * vh::kMlpParams));
  MLP_CUDA(cudaMemset(m->v, 0, sizeof(float) * vh::kMlpParams));
  m->steps = 0;
  vh::launch_mlp_pack(m->P, m->packed, 0);
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaDeviceSynchronize());
  return VH_OK;
}

vh_status vh_mlp_get_params(vh_mlp* m, float* host) {
  if (!m || !host) return mlp_fail(VH_ERR_ARG, "vh_mlp_get_params: NULL argument");
  MLP_CUDA(cudaSetDevice(m->device));
  MLP_CUDA(cudaMemcpy(host, m->P, sizeof(float) * vh::kMlpParams, cudaMemcpyDeviceToHost));
  return VH_OK;
}

vh_status vh_mlp_create(int device, unsigned long long seed, vh_mlp** out) {
  if (!out) return mlp_fail(VH_ERR_ARG, "vh_mlp_create: out is NULL");
  *out = nullptr;
  MLP_CUDA(cudaSetDevice(device));
  vh_mlp* m = new vh_mlp;
  m->device = device;
  const size_t b = sizeof(float) * vh::kMlpParams;
  cudaError_t e;
  if ((e = cudaMalloc(&m->P, b)) || (e = cudaMalloc(&m->G, b)) || (e = cudaMalloc(&m->m, b)) ||
      (e = cudaMalloc(&m->v, b)) || (e = cudaMalloc(&m->loss, sizeof(float))) ||
      (e = cudaMalloc(&m->packed, sizeof(uint32_t) * vh::mlp_pack_words()))) {
    vh_mlp_destroy(m);
    return mlp_cuda(e, "vh_mlp_create: cudaMalloc");
  }
  // Glorot-uniform weights, zero biases (|v| bias at 0.5)
  std::vector<float> h(vh::kMlpParams, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_out, int fan_in) {
    const float a = std::sqrt(6.f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> u(-a, a);
    for (int i = 0; i < fan_out * fan_in; i++) h[off + i] = u(rng);
  };
  fill(vh::kW1, 64, 4);
  fill(vh::kW2, 64, 64);
  fill(vh::kW3, 3, 64);
  h[vh::kB3 + 1] = 0.5f;
  vh_status st = vh_mlp_set_params(m, h.data());
  if (st != VH_OK) {
    vh_mlp_destroy(m);
    return st;
  }
  *out = m;
  return VH_OK;
}

vh_status vh_mlp_forward(vh_mlp* m, const float* X, long n, float* Y) {
  if (!m || n < 0 || (n > 0 && (!X || !Y))) return mlp_fail(VH_ERR_ARG, "vh_mlp_forward: bad arguments");
  MLP_CUDA(cudaSetDevice(m->device));
  vh::launch_mlp_forward(m->packed, X, n, Y, 0);
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaDeviceSynchronize());
  return VH_OK;
}

vh_status vh_mlp_grad(vh_mlp* m, const float* X, const float* Y, long n, float* grad, float* loss) {
  if (!m || n <= 0 || !X || !Y || !grad) return mlp_fail(VH_ERR_ARG, "vh_mlp_grad: bad arguments");
  MLP_CUDA(cudaSetDevice(m->device));
  MLP_CUDA(cudaMemset(m->G, 0, sizeof(float) * vh::kMlpParams));
  MLP_CUDA(cudaMemset(m->loss, 0, sizeof(float)));
  MLP_CUDA(vh::launch_mlp_grad(m->P, X, Y, n, 0, 1, n, m->G, m->loss, 0));
  MLP_CUDA(cudaMemcpy(grad, m->G, sizeof(float) * vh::kMlpParams, cudaMemcpyDeviceToHost));
  float l = 0.f;
  MLP_CUDA(cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) *loss = l / (float)n;
  return VH_OK;
}

vh_status vh_mlp_train(vh_mlp* m, const float* X, const float* Y, long n, int batch, int epochs,
                       float lr, unsigned long long seed, float* epoch_loss) {
  if (!m || !X || !Y || n <= 0 || batch <= 0 || epochs <= 0 || !(lr > 0.f))
    return mlp_fail(VH_ERR_ARG, "vh_mlp_train: bad arguments");
  MLP_CUDA(cudaSetDevice(m->device));
  std::mt19937_64 rng(seed);
  const long long iters = (n + batch - 1) / batch, total = iters * (long long)epochs;
  long long k = 0;
  for (int ep = 0; ep < epochs; ep++) {
    // a full permutation of the samples: idx(b) = (off + b * stride) mod n
    long long stride = 1;
    if (n > 1) {
      do {
        stride = 1 + (long long)(rng() % (unsigned long long)(n - 1));
      } while (gcdll(stride, n) != 1);
    }
    const long long off0 = (long long)(rng() % (unsigned long long)n);
    MLP_CUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), 0));
    for (long long it = 0; it < iters; it++, k++) {
      const long long b0 = it * batch, cnt = std::min<long long>(batch, n - b0);
      const long long off = (long long)((off0 + (unsigned long long)(b0 % n) * (unsigned long long)stride) % (unsigned long long)n);
      MLP_CUDA(cudaMemsetAsync(m->G, 0, sizeof(float) * vh::kMlpParams, 0));
      MLP_CUDA(vh::launch_mlp_grad(m->P, X, Y, n, off, stride, cnt, m->G, m->loss, 0));
      m->steps++;
      const float lrk = lr * 0.5f * (1.f + std::cos(3.14159265f * (float)k / (float)total));
      const float b1c = 1.f - std::pow(0.9f, (float)m->steps);
      const float b2c = 1.f - std::pow(0.999f, (float)m->steps);
      vh::launch_mlp_adam(m->P, m->G, m->m, m->v, lrk, b1c, b2c, 0);
      MLP_CUDA(cudaGetLastError());
    }
    if (epoch_loss) {
      float l = 0.f;
      MLP_CUDA(cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
      epoch_loss[ep] = l / (float)n;
    }
  }
  vh::launch_mlp_pack(m->P, m->packed, 0);
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaDeviceSynchronize());
  return VH_OK;
}

}  // extern "C"
