// vh_mlp.cuh -- the learned con2prim start point (vh_mlp.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vh_physics.cuh"

namespace vh {

// 4 -> 64 -> 64 -> 3: W1[64][4], b1[64], W2[64][64], b2[64], W3[3][64], b3[3]
constexpr int kMlpParams = 4675;

int mlp_pack_words();
size_t mlp_grad_smem();
void launch_mlp_pack(const float* P, uint32_t* packed, cudaStream_t s);
void launch_mlp_forward(const uint32_t* W, const float* X, long long n, float* Y, cudaStream_t s);
// tau from the device clock clk[0]
void launch_mlp_guess(const uint32_t* W, const double* Q, long long N, const double* clk, float* vg,
                      cudaStream_t s);
void launch_mlp_samples(const EosDev& E, const double* Q, long long N, double tau, float* X,
                        float* Y, long long cap, unsigned long long* count, cudaStream_t s);
cudaError_t launch_mlp_grad(const float* P, const float* X, const float* Y, long long n,
                            long long off, long long stride, long long cnt, float* G, float* loss,
                            cudaStream_t s);
void launch_mlp_adam(float* P, const float* G, float* m, float* v, float lr, float b1c, float b2c,
                     cudaStream_t s);

}  // namespace vh

// the network object behind the C ABI's opaque vh_mlp
struct vh_mlp {
  int device = 0;
  float* P = nullptr;  // FP32 master parameters [kMlpParams]
  float* G = nullptr;  // gradients
  float* m = nullptr;  // Adam moments
  float* v = nullptr;
  float* loss = nullptr;
  uint32_t* packed = nullptr;  // BF16 inference weights
  long long steps = 0;         // Adam steps taken
};
