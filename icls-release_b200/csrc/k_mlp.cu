// k_mlp.cu — the learned interface curvature: a 27-128-128-64-1 SiLU MLP
// on tcgen05 tensor-core tiles (BF16 operands, FP32 accumulation in tensor
// memory).  Compiled without -fmad=false: this is not reference arithmetic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "../../include/icls_gpu.h"
#include "batch.cuh"
#include "umma.cuh"

namespace icls {
namespace {

using umma::kmajor_off;
using umma::kRows;

// ---- one 128 x n tile product, a check of the tensor-core path ----------
// a: 128 x k row-major BF16, b: n x k row-major BF16, d: 128 x n FP32
__global__ void __launch_bounds__(128) k_tc_gemm_check(const __nv_bfloat16* __restrict__ a,
                                                       const __nv_bfloat16* __restrict__ b, float* __restrict__ d,
                                                       int n, int k, int* __restrict__ err) {
  // 16-byte alignment is all the no-swizzle layout needs (a larger __align__ on
  // dynamic shared memory is not honoured in relocatable-device-code builds)
  extern __shared__ __align__(16) unsigned char dyn[];
  __nv_bfloat16* sa = reinterpret_cast<__nv_bfloat16*>(dyn);                       // 128 x 128 max
  __nv_bfloat16* sb = reinterpret_cast<__nv_bfloat16*>(dyn + kRows * 128 * 2);     // 128 x 128 max
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, warp = t >> 5;
  for (int e = t; e < kRows * k; e += blockDim.x) {
    const int r = e / k, kk = e - r * k;
    *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(sa) + kmajor_off(r, kk, kRows)) = a[e];
  }
  for (int e = t; e < n * k; e += blockDim.x) {
    const int r = e / k, kk = e - r * k;
    *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(sb) + kmajor_off(r, kk, n)) = b[e];
  }
  if (t == 0) umma::mbar_init(&bar, 1);
  if (warp == 0) umma::tmem_alloc(&tmem_slot, 128);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tmem_slot;
  uint32_t phase = 0;
  const bool ok = umma::tile_gemm(sa, sb, n, k, tmem, &bar, phase);
  if (!ok) {
    if (t == 0) atomicExch(err, 1);
    umma::mbar_wait(&bar, phase ^ 1u);  // let a late completion land before the columns are freed
  } else {
    for (int c = 0; c < n; c += 8) {
      float v[8];
      umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
#pragma unroll
      for (int q = 0; q < 8; ++q) d[t * n + c + q] = v[q];
    }
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, 128);
}


// ============================================================== the network
// 27 -> 128 -> 128 -> 64 -> 1, SiLU after the first three layers.  Inputs
// are the features of the 27 values (phi(x + o dx) - phi(x)) / dx of a
// 3x3x3 stencil (mlp_features: its second-order part and unit gradient,
// 30 values padded to 32), the output is the correction to the plain stencil's
// kappa * dx: the learned curvature is kappa_stencil + output / dx, so a
// well-resolved interface, where the stencil is already accurate, needs
// only a small output.  FP32 master parameters in one
// array (layout below), BF16 copies of W1..W3 as the tiles' B operands and
// BF16 transposes of W2, W3 for back-propagation to the inputs.
constexpr int kIn = 32, kH1 = 128, kH2 = 128, kH3 = 64;
// layer 1 takes each FP32 input as a BF16 pair hi + lo (K = 2 x 32) against
// W1 twice: the inputs' small second differences, which carry the
// curvature, keep about 16 mantissa bits
constexpr int kIn2 = 2 * kIn;
constexpr int oW1 = 0, oB1 = oW1 + kH1 * kIn, oW2 = oB1 + kH1, oB2 = oW2 + kH2 * kH1, oW3 = oB2 + kH2,
              oB3 = oW3 + kH3 * kH2, oW4 = oB3 + kH3, oB4 = oW4 + kH3, kParams = oB4 + 1;

struct Net {
  const float* theta;              // FP32 parameters
  const __nv_bfloat16* w1;         // [128][64] = [W1 | W1]
  const __nv_bfloat16* w2;         // [128][128]
  const __nv_bfloat16* w3;         // [64][128]
  const __nv_bfloat16* w2t;        // [128][128] = W2^T
  const __nv_bfloat16* w3t;        // [128][64]  = W3^T
};

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}
__device__ __forceinline__ void put_bf16(unsigned char* base, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16(v);
}

// shared-memory plan of one tile (bytes)
constexpr int SB_B = 0;                       // weight operand, up to 128 x 128
constexpr int SB_ACT = SB_B + 32768;          // activations / deltas, A layout [128 x 128]
constexpr int SB_XA = SB_ACT + 32768;         // inputs hi|lo, A layout [128 x 64]
constexpr int SB_XT = SB_XA + 16384;          // inputs transposed [64 x 128]
constexpr int SB_H1T = SB_XT + 16384;         // H1^T [128 x 128]
constexpr int SB_H2T = SB_H1T + 32768;        // H2^T [128 x 128]
constexpr int SB_DZT = SB_H2T + 32768;        // delta^T [128 x 128]
constexpr int SB_TRAIN = SB_DZT + 32768;      // 196608

// a weight matrix [n][k] (row-major BF16, global) into the B operand layout
__device__ __forceinline__ void stage_b(unsigned char* sb, const __nv_bfloat16* __restrict__ w, int n, int k) {
  for (int e = threadIdx.x; e < n * k; e += blockDim.x) {
    const int r = e / k, c = e - r * k;
    *reinterpret_cast<__nv_bfloat16*>(sb + kmajor_off(r, c, n)) = w[e];
  }
}

// The forward pass of one 128-sample tile; x (FP32, [rows][32]) holds the
// tile's inputs, sample t of the tile is row t.  Returns y (kappa*dx) of this
// thread's sample.  Training keeps the pre-activations z1..z3 (zg, per sample
// 320 floats) and the transposed activations in shared memory.
template <bool TRAIN>
__device__ float forward_tile(const Net& net, const float* __restrict__ xrow, unsigned char* sm, uint32_t tmem,
                              uint64_t* bar, uint32_t& phase, float* __restrict__ zrow, bool& ok) {
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  // inputs
  for (int j = 0; j < kIn; ++j) {
    const float v = xrow ? xrow[j] : 0.f;
    const float hi = __bfloat162float(__float2bfloat16(v));
    const float lo = v - hi;
    put_bf16(sm + SB_XA, kmajor_off(t, j, kRows), hi);
    put_bf16(sm + SB_XA, kmajor_off(t, j + kIn, kRows), lo);
    if (TRAIN) {
      put_bf16(sm + SB_XT, kmajor_off(j, t, kIn2), hi);
      put_bf16(sm + SB_XT, kmajor_off(j + kIn, t, kIn2), lo);
    }
  }
  // layer 1
  stage_b(sm + SB_B, net.w1, kH1, kIn2);
  ok &= umma::tile_gemm(sm + SB_XA, sm + SB_B, kH1, kIn2, tmem, bar, phase);
  for (int c = 0; c < kH1; c += 8) {
    float v[8];
    umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float z = v[q] + net.theta[oB1 + c + q];
      const float h = silu(z);
      put_bf16(sm + SB_ACT, kmajor_off(t, c + q, kRows), h);
      if (TRAIN) {
        put_bf16(sm + SB_H1T, kmajor_off(c + q, t, kH1), h);
        zrow[c + q] = z;
      }
    }
  }
  // layer 2
  stage_b(sm + SB_B, net.w2, kH2, kH1);
  ok &= umma::tile_gemm(sm + SB_ACT, sm + SB_B, kH2, kH1, tmem, bar, phase);
  for (int c = 0; c < kH2; c += 8) {
    float v[8];
    umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float z = v[q] + net.theta[oB2 + c + q];
      const float h = silu(z);
      put_bf16(sm + SB_ACT, kmajor_off(t, c + q, kRows), h);
      if (TRAIN) {
        put_bf16(sm + SB_H2T, kmajor_off(c + q, t, kH2), h);
        zrow[kH1 + c + q] = z;
      }
    }
  }
  // layer 3 and the linear head
  stage_b(sm + SB_B, net.w3, kH3, kH2);
  ok &= umma::tile_gemm(sm + SB_ACT, sm + SB_B, kH3, kH2, tmem, bar, phase);
  float y = net.theta[oB4];
  for (int c = 0; c < kH3; c += 8) {
    float v[8];
    umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float z = v[q] + net.theta[oB3 + c + q];
      y += net.theta[oW4 + c + q] * silu(z);
      if (TRAIN) zrow[kH1 + kH2 + c + q] = z;
    }
  }
  return y;
}

// warp-summed atomic add of this thread's v into *dst (one atomic per warp)
__device__ __forceinline__ void warp_add(float* dst, float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
}

// One training tile: forward, weighted squared-error gradient (dy = scale x
// weight x error, scale = 2/batch; no weights: 1) and the backward pass; parameter gradients are added into grad (FP32), the loss
// sum into *loss.  Samples idx = (a * (base + t) + b) mod n (a per-epoch
// affine shuffle of the n samples, n a power of two, a odd).
__global__ void __launch_bounds__(128) k_mlp_train_tile(Net net, const float* __restrict__ X,
                                                        const float* __restrict__ label,
                                                        const float* __restrict__ weight, long long n, long long base,
                                                        unsigned long long pa, unsigned long long pb, float scale,
                                                        float* __restrict__ zbuf, float* __restrict__ grad,
                                                        float* __restrict__ loss, int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, warp = t >> 5;
  if (t == 0) umma::mbar_init(&bar, 1);
  if (warp == 0) umma::tmem_alloc(&tmem_slot, 128);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  const long long gi = base + (long long)blockIdx.x * kRows + t;
  const long long s = (long long)(((unsigned long long)gi * pa + pb) & (unsigned long long)(n - 1));
  float* zrow = zbuf + ((long long)blockIdx.x * kRows + t) * (kH1 + kH2 + kH3);
  const float y = forward_tile<true>(net, X + s * kIn, sm, tmem, &bar, phase, zrow, ok);
  const float e = y - label[s];
  const float wt = weight ? weight[s] : 1.f;
  warp_add(loss, wt * e * e);
  const float dy = scale * wt * e;
  // head: dW4 = sum dy h3, db4 = sum dy; delta3 = dy W4 silu'(z3)
  warp_add(grad + oB4, dy);
  for (int j = 0; j < kH3; ++j) {
    const float z = zrow[kH1 + kH2 + j];
    warp_add(grad + oW4 + j, dy * silu(z));
    const float d3 = dy * net.theta[oW4 + j] * dsilu(z);
    warp_add(grad + oB3 + j, d3);
    put_bf16(sm + SB_ACT, kmajor_off(t, j, kRows), d3);
    put_bf16(sm + SB_DZT, kmajor_off(j, t, kRows), d3);
    put_bf16(sm + SB_DZT, kmajor_off(j + kH3, t, kRows), 0.f);  // rows 64..127 of delta3^T are padding
  }
  // dW3 = delta3^T H2 (rows 0..63 of a 128 x 128 tile)
  ok &= umma::tile_gemm(sm + SB_DZT, sm + SB_H2T, kH2, kRows, tmem, &bar, phase);
  if (t < kH3)
    for (int c = 0; c < kH2; c += 8) {
      float v[8];
      umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
      for (int q = 0; q < 8; ++q) atomicAdd(grad + oW3 + t * kH2 + c + q, v[q]);
    }
  else
    for (int c = 0; c < kH2; c += 8) {  // every lane of the warp takes part in tcgen05.ld
      float v[8];
      umma::tmem_ld8(lane_addr + c, v);
    }
  // dH2 = delta3 W3 -> delta2 = dH2 silu'(z2)
  stage_b(sm + SB_B, net.w3t, kH2, kH3);
  ok &= umma::tile_gemm(sm + SB_ACT, sm + SB_B, kH2, kH3, tmem, &bar, phase);
  for (int c = 0; c < kH2; c += 8) {
    float v[8];
    umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float d2 = v[q] * dsilu(zrow[kH1 + c + q]);
      warp_add(grad + oB2 + c + q, d2);
      put_bf16(sm + SB_ACT, kmajor_off(t, c + q, kRows), d2);
      put_bf16(sm + SB_DZT, kmajor_off(c + q, t, kRows), d2);
    }
  }
  // dW2 = delta2^T H1
  ok &= umma::tile_gemm(sm + SB_DZT, sm + SB_H1T, kH1, kRows, tmem, &bar, phase);
  for (int c = 0; c < kH1; c += 8) {
    float v[8];
    umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) atomicAdd(grad + oW2 + t * kH1 + c + q, v[q]);
  }
  // dH1 = delta2 W2 -> delta1
  stage_b(sm + SB_B, net.w2t, kH1, kH2);
  ok &= umma::tile_gemm(sm + SB_ACT, sm + SB_B, kH1, kH2, tmem, &bar, phase);
  for (int c = 0; c < kH1; c += 8) {
    float v[8];
    umma::tmem_ld8(lane_addr + c, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float d1 = v[q] * dsilu(zrow[c + q]);
      warp_add(grad + oB1 + c + q, d1);
      put_bf16(sm + SB_DZT, kmajor_off(c + q, t, kRows), d1);
    }
  }
  // dW1 = delta1^T X (the hi and lo halves both act through W1)
  ok &= umma::tile_gemm(sm + SB_DZT, sm + SB_XT, kIn2, kRows, tmem, &bar, phase);
  for (int c = 0; c < kIn; c += 8) {
    float v[8], w[8];
    umma::tmem_ld8(lane_addr + c, v);
    umma::tmem_ld8(lane_addr + kIn + c, w);
#pragma unroll
    for (int q = 0; q < 8; ++q) atomicAdd(grad + oW1 + t * kIn + c + q, v[q] + w[q]);
  }
  if (!ok && t == 0) atomicExch(err, 1);
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, 128);
}

// ---- inference with the weights resident in shared memory --------------
// A persistent CTA stages W1..W3 (B operands) and the biases once and then
// runs its 128-sample tiles back to back.  The first 16 KB of the
// activation buffer also hold a tile's inputs (hi | lo, A layout [128 x 64]):
// layer 1 has finished reading them before its epilogue writes the first
// activations.  99,856 bytes: two CTAs per SM.
constexpr int SI_W1 = 0;                          // [128 x 64]
constexpr int SI_W2 = SI_W1 + kH1 * kIn2 * 2;     // [128 x 128]
constexpr int SI_W3 = SI_W2 + kH2 * kH1 * 2;      // [64 x 128]
constexpr int SI_ACT = SI_W3 + kH3 * kH2 * 2;     // [128 x 128], inputs in its first 16 KB
constexpr int SI_PAR = SI_ACT + kRows * kH1 * 2;  // b1, b2, b3, w4, b4 (FP32)
constexpr int PB1 = 0, PB2 = PB1 + kH1, PB3 = PB2 + kH2, PW4 = PB3 + kH3, PB4 = PW4 + kH3;
constexpr int SB_INFER = SI_PAR + 4 * (PB4 + 4);

// SiLU for the forward-only path (the BF16 rounding that follows dwarfs the
// approximate divide); the exponent is capped so the divisor stays finite
__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.f + __expf(fminf(-z, 80.f))); }
// SiLU of a hidden activation that is stored as BF16 next: z sigma(z) with
// sigma(z) = (1 + tanh(z/2))/2, so z (1 + tanh(z/2))/2 = h + h tanh(h) for
// h = z/2, on the hardware tanh (tanh.approx.f32, absolute error about
// 2^-11): one transcendental instead of an exponential and a reciprocal,
// with an error below the BF16 rounding (2^-9 relative) that follows
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu_bf16(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_hw(h), h);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a at the lower address
  return *reinterpret_cast<const uint32_t*>(&h);
}

// a weight matrix [n][k] (row-major BF16, 16-byte aligned rows) into the
// B-operand layout, one 16-byte chunk per store
__device__ __forceinline__ void stage_rows(unsigned char* dst, const __nv_bfloat16* __restrict__ w, int n, int k) {
  for (int e = threadIdx.x; e < n * (k / 8); e += blockDim.x) {
    const int c = e / n, r = e - c * n;
    *reinterpret_cast<uint4*>(dst + kmajor_off(r, 8 * c, n)) =
        *reinterpret_cast<const uint4*>(w + (size_t)r * k + 8 * c);
  }
}

// row t of the tile: the sample's 32 FP32 inputs (from registers; zeros
// past the end) as BF16 hi (k 0..31) and lo (k 32..63)
__device__ __forceinline__ void stage_inputs_regs(unsigned char* act, const float4 (&xv)[kIn / 4], int t) {
#pragma unroll
  for (int c = 0; c < kIn / 8; ++c) {
    const float4 a = xv[2 * c], b = xv[2 * c + 1];
    const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    float hi[8], lo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      hi[q] = __bfloat162float(__float2bfloat16(v[q]));
      lo[q] = v[q] - hi[q];
    }
    *reinterpret_cast<uint4*>(act + kmajor_off(t, 8 * c, kRows)) =
        make_uint4(pack_bf16(hi[0], hi[1]), pack_bf16(hi[2], hi[3]), pack_bf16(hi[4], hi[5]), pack_bf16(hi[6], hi[7]));
    *reinterpret_cast<uint4*>(act + kmajor_off(t, kIn + 8 * c, kRows)) =
        make_uint4(pack_bf16(lo[0], lo[1]), pack_bf16(lo[2], lo[3]), pack_bf16(lo[4], lo[5]), pack_bf16(lo[6], lo[7]));
  }
}

// a hidden layer's epilogue: row t of SiLU(D + bias) as the next A operand
__device__ __forceinline__ void hidden_epilogue(uint32_t lane_addr, const float* bias, int n, unsigned char* act,
                                                int t) {
  for (int c0 = 0; c0 < n; c0 += 32) {
    float v[32];
    umma::tmem_ld32(lane_addr + (uint32_t)c0, v);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      float h[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) h[q] = silu_bf16(v[8 * m + q] + bias[c0 + 8 * m + q]);
      *reinterpret_cast<uint4*>(act + kmajor_off(t, c0 + 8 * m, kRows)) =
          make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
    }
  }
}

// The forward pass over samples 0..n-1 of X (FP32 [n][32], 16-byte
// aligned), tiles blockIdx.x, blockIdx.x + gridDim.x, ...; out.begin(s,
// live) is called when a tile starts (what the output step will need can be
// read then) and out(s, y) takes each sample's output.  The next tile's
// inputs are read while the current tile runs.  All 128 threads call it.
template <class Out>
__device__ __forceinline__ void infer_tiles(const Net& net, const float* __restrict__ X, long long n, Out& out,
                                            int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, warp = t >> 5;
  const long long tiles = (n + kRows - 1) / kRows;
  if ((long long)blockIdx.x >= tiles) return;  // block-uniform: no tensor memory taken
  stage_rows(sm + SI_W1, net.w1, kH1, kIn2);
  stage_rows(sm + SI_W2, net.w2, kH2, kH1);
  stage_rows(sm + SI_W3, net.w3, kH3, kH2);
  float* par = reinterpret_cast<float*>(sm + SI_PAR);
  for (int e = t; e < kH1; e += blockDim.x) par[PB1 + e] = net.theta[oB1 + e];
  for (int e = t; e < kH2; e += blockDim.x) par[PB2 + e] = net.theta[oB2 + e];
  for (int e = t; e < kH3; e += blockDim.x) {
    par[PB3 + e] = net.theta[oB3 + e];
    par[PW4 + e] = net.theta[oW4 + e];
  }
  if (t == 0) {
    par[PB4] = net.theta[oB4];
    umma::mbar_init(&bar, 1);
  }
  if (warp == 0) umma::tmem_alloc(&tmem_slot, 128);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  float4 xv[kIn / 4];
  auto load_x = [&](long long s) {
#pragma unroll
    for (int q = 0; q < kIn / 4; ++q)
      xv[q] = s < n ? reinterpret_cast<const float4*>(X + s * kIn)[q] : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  load_x((long long)blockIdx.x * kRows + t);
  for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const long long s = tile * kRows + t;
    out.begin(s, s < n);
    stage_inputs_regs(sm + SI_ACT, xv, t);
    load_x(s + (long long)gridDim.x * kRows);  // in flight during this tile
    ok &= umma::tile_gemm(sm + SI_ACT, sm + SI_W1, kH1, kIn2, tmem, &bar, phase);
    hidden_epilogue(lane_addr, par + PB1, kH1, sm + SI_ACT, t);
    ok &= umma::tile_gemm(sm + SI_ACT, sm + SI_W2, kH2, kH1, tmem, &bar, phase);
    hidden_epilogue(lane_addr, par + PB2, kH2, sm + SI_ACT, t);
    ok &= umma::tile_gemm(sm + SI_ACT, sm + SI_W3, kH3, kH2, tmem, &bar, phase);
    float y = par[PB4];
    for (int c0 = 0; c0 < kH3; c0 += 32) {
      float v[32];
      umma::tmem_ld32(lane_addr + (uint32_t)c0, v);
#pragma unroll
      for (int q = 0; q < 32; ++q) y += par[PW4 + c0 + q] * silu_fast(v[q] + par[PB3 + c0 + q]);
    }
    if (s < n) out(s, y);
    if (!__syncthreads_and(ok)) break;  // block-uniform exit after a wait that gave up
  }
  if (!ok) {
    if (t == 0) atomicExch(err, 1);
    umma::mbar_wait(&bar, phase ^ 1u);  // let a late completion land before the columns are freed
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, 128);
}

struct StoreOut {
  float* y;
  __device__ void begin(long long, bool) {}
  __device__ void operator()(long long s, float v) const { y[s] = v; }
};

// inference over n samples into y
__global__ void __launch_bounds__(128, 2) k_mlp_infer(Net net, const float* __restrict__ X, long long n,
                                                      float* __restrict__ y, int* __restrict__ err) {
  StoreOut o{y};
  infer_tiles(net, X, n, o, err);
}

// parameter q's BF16 value into the tile copies
__device__ __forceinline__ void put_copies(int q, __nv_bfloat16 h, __nv_bfloat16* w1, __nv_bfloat16* w2,
                                           __nv_bfloat16* w3, __nv_bfloat16* w2t, __nv_bfloat16* w3t) {
  if (q >= oW1 && q < oB1) {
    const int r = (q - oW1) / kIn, c = (q - oW1) % kIn;
    w1[r * kIn2 + c] = h;
    w1[r * kIn2 + kIn + c] = h;
  }
  if (q >= oW2 && q < oB2) {
    const int r = (q - oW2) / kH1, c = (q - oW2) % kH1;
    w2[q - oW2] = h;
    w2t[c * kH2 + r] = h;
  }
  if (q >= oW3 && q < oB3) {
    const int r = (q - oW3) / kH2, c = (q - oW3) % kH2;
    w3[q - oW3] = h;
    w3t[c * kH3 + r] = h;
  }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 parameters, then the
// BF16 copies and transposes; the gradient is cleared for the next batch
__global__ void k_mlp_adam(float* __restrict__ theta, float* __restrict__ grad, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float bc1, float bc2, __nv_bfloat16* __restrict__ w1,
                           __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w3,
                           __nv_bfloat16* __restrict__ w2t, __nv_bfloat16* __restrict__ w3t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kParams) return;
  const float g = grad[q];
  grad[q] = 0.f;
  const float a = 0.9f * m1[q] + 0.1f * g;
  const float b = 0.999f * m2[q] + 0.001f * g * g;
  m1[q] = a;
  m2[q] = b;
  const float w = theta[q] - lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
  theta[q] = w;
  const __nv_bfloat16 h = __float2bfloat16(w);
  put_copies(q, h, w1, w2, w3, w2t, w3t);
}

// refresh the BF16 copies from theta (after initialisation or a set)
__global__ void k_mlp_copies(const float* __restrict__ theta, __nv_bfloat16* __restrict__ w1,
                             __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w3,
                             __nv_bfloat16* __restrict__ w2t, __nv_bfloat16* __restrict__ w3t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kParams) return;
  put_copies(q, __float2bfloat16(theta[q]), w1, w2, w3, w2t, w3t);
}

// ===================================================== training samples
// counter-based uniform in [0,1) (splitmix64 of seed, sample and draw)
__device__ __forceinline__ double urand(unsigned long long seed, unsigned long long i, unsigned long long d) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i * 64ull + d + 1ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

__constant__ double cPu[270];  // the least-squares pseudo-inverse for unit spacing
__constant__ float cPuf[270];  // the same rounded to FP32 (the FP32 features)
template <typename R>
__device__ __forceinline__ R cpu_coef(int q) {
  if constexpr (sizeof(R) == 4) return cPuf[q];
  else return (R)cPu[q];
}

// The network's inputs from a stencil f (phi(x + o) - phi(x), in cells,
// o in {-1,0,1}^3 with z outer): the stencil minus its least-squares linear
// part g.o (27 values, the second-order part that carries the curvature),
// then the unit gradient g/|g| (3 values) and 2 zeros.  Removing the linear
// part before the BF16 tiles keeps their rounding far below the curvature
// signal.
template <typename R>
__device__ __forceinline__ void mlp_features(const R* f, float* out) {
  R g[3] = {0, 0, 0};
  for (int q = 0; q < 27; ++q)
    for (int r = 1; r <= 3; ++r) g[r - 1] += cpu_coef<R>(r * 27 + q) * f[q];
  int q = 0;
  for (int dk = -1; dk <= 1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di, ++q) out[q] = (float)(f[q] - (g[0] * di + g[1] * dj + g[2] * dk));
  const R n = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  const R rn = n > (R)0 ? (R)1 / n : (R)0;
  out[27] = (float)(g[0] * rn);
  out[28] = (float)(g[1] * rn);
  out[29] = (float)(g[2] * rn);
  out[30] = 0.f;
  out[31] = 0.f;
}

struct Shape {
  double c[3];   // centre
  double s[3];   // semi-axes (a sphere has three equal)
  double R[9];   // body-to-world rotation, column-major
  int sphere;
};

// signed distance to the shape (outside > 0); for an ellipsoid by bisection
// on the Lagrange multiplier of the closest-point problem
__device__ double sdist(const Shape& S, const double* x, double* foot) {
  double d[3] = {x[0] - S.c[0], x[1] - S.c[1], x[2] - S.c[2]};
  if (S.sphere) {
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    return r - S.s[0];
  }
  double y[3];
  for (int i = 0; i < 3; ++i) y[i] = S.R[0 + 3 * i] * d[0] + S.R[1 + 3 * i] * d[1] + S.R[2 + 3 * i] * d[2];
  double g = 0.;
  for (int i = 0; i < 3; ++i) g += y[i] * y[i] / (S.s[i] * S.s[i]);
  const bool outside = g > 1.;
  const double smin = fmin(S.s[0], fmin(S.s[1], S.s[2]));
  auto F = [&](double t) {
    double f = 0.;
    for (int i = 0; i < 3; ++i) {
      const double q = S.s[i] * y[i] / (S.s[i] * S.s[i] + t);
      f += q * q;
    }
    return f - 1.;
  };
  double lo, hi;
  if (outside) {
    lo = 0.;
    hi = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]) * fmax(S.s[0], fmax(S.s[1], S.s[2])) + 1.;
  } else {
    lo = -smin * smin;
    hi = 0.;
  }
  for (int it = 0; it < 200; ++it) {  // F decreases in t on the bracket
    const double mid = 0.5 * (lo + hi);
    if (F(mid) > 0.) lo = mid;
    else hi = mid;
    if (hi - lo <= 1e-15 * fmax(1., fabs(mid))) break;
  }
  const double t = 0.5 * (lo + hi);
  double q[3], dd = 0.;
  for (int i = 0; i < 3; ++i) {
    q[i] = S.s[i] * S.s[i] * y[i] / (S.s[i] * S.s[i] + t);
    dd += (y[i] - q[i]) * (y[i] - q[i]);
  }
  if (foot)
    for (int i = 0; i < 3; ++i) foot[i] = q[i];
  return outside ? sqrt(dd) : -sqrt(dd);
}

// least-squares curvature of a 3x3x3 stencil f (order z-outer, x-inner) of
// spacing h (interface.f90:57-111 without its clamps)
__device__ double lsq_curv(const double* f, double h) {
  double x[10];
  for (int r = 1; r < 10; ++r) {
    double acc = 0.;
    for (int q = 0; q < 27; ++q) acc += cPu[r * 27 + q] * f[q];
    x[r] = acc;
  }
  for (int r = 1; r <= 3; ++r) x[r] /= h;
  for (int r = 4; r <= 9; ++r) x[r] /= h * h;
  const double nv = sqrt(x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
  const double n3 = nv * nv * nv;
  const double t1 = (x[4] + x[5] + x[6]) / nv;
  const double t2 = (x[1] * x[1] * x[4] + x[2] * x[2] * x[5] + x[3] * x[3] * x[6]) / n3;
  const double t3 = 2. * (x[1] * x[2] * x[7] + x[1] * x[3] * x[8] + x[2] * x[3] * x[9]) / n3;
  return -((t1 - t2) - t3);
}

// principal curvatures k1 >= k2 of an ellipsoid at the surface point q
// (body frame), positive where convex
__device__ void ellipsoid_principal(const Shape& S, const double* q, double& k1, double& k2) {
  double g[3], gn = 0.;
  for (int i = 0; i < 3; ++i) {
    g[i] = 2. * q[i] / (S.s[i] * S.s[i]);
    gn += g[i] * g[i];
  }
  gn = sqrt(gn);
  double n[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
  // M = P H P / |g| with H = diag(2/s^2), P = I - n n^T: eigenvalues 0, k1, k2
  double M[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.;
      for (int k = 0; k < 3; ++k) {
        const double Pik = (i == k ? 1. : 0.) - n[i] * n[k];
        const double Pkj = (k == j ? 1. : 0.) - n[k] * n[j];
        acc += Pik * (2. / (S.s[k] * S.s[k])) * Pkj;
      }
      M[i][j] = acc / gn;
    }
  const double T = M[0][0] + M[1][1] + M[2][2];
  double T2 = 0.;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T2 += M[i][j] * M[j][i];
  const double Q = 0.5 * (T * T - T2);
  const double disc = fmax(0.25 * T * T - Q, 0.);
  k1 = 0.5 * T + sqrt(disc);
  k2 = 0.5 * T - sqrt(disc);
}

// Sample i: a seeded sphere (R in [3,40] cells) or ellipsoid (semi-axes in
// [4,40] cells, random rotation) on a unit grid, a grid node x with
// |phi(x)| <= 3 near its surface, phi the exact signed distance.  Writes the
// 27 inputs (phi(x+o) - phi(x), o in {-1,0,1}^3), the label (the
// least-squares curvature of the stencil of spacing 1/4 at x, the method on a
// grid refined 4x, minus the plain curvature at spacing 1) and, in extra,
// the plain curvature at spacing 1, the analytic curvature and the shape's
// smallest radius.
__global__ void k_mlp_gen(unsigned long long seed, long long n, float* __restrict__ X,
                          float* __restrict__ label, float* __restrict__ weight, float* __restrict__ extra) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double pi2 = 6.283185307179586;
  Shape S;
  double x[3] = {0., 0., 0.}, kana = 0., lab = 0., ff[27];
  int d = 0;
  // Draw shapes and points until the node is near the surface (|phi| <= 3)
  // and the level set through it is resolved: curvature radius of at least 3
  // cells (|kappa dx| <= 2/3), the focal points more than two cells further
  // in (1 + k_i (phi - 2) >= 1/2), and the refined-grid label within 0.02 of
  // the exact curvature (its stencil does not straddle a kink of the signed
  // distance).
  for (int tries = 0; tries < 256; ++tries) {
    S.sphere = urand(seed, i, d++) < 0.5;
    for (int k = 0; k < 3; ++k) S.c[k] = urand(seed, i, d++);
    if (S.sphere) {
      const double R = 3. + 37. * urand(seed, i, d++);
      S.s[0] = S.s[1] = S.s[2] = R;
    } else {
      for (int k = 0; k < 3; ++k) S.s[k] = 4. + 36. * urand(seed, i, d++);
      const double u1 = urand(seed, i, d++), u2 = urand(seed, i, d++), u3 = urand(seed, i, d++);
      const double qx = sqrt(1. - u1) * sin(pi2 * u2), qy = sqrt(1. - u1) * cos(pi2 * u2);
      const double qz = sqrt(u1) * sin(pi2 * u3), qw = sqrt(u1) * cos(pi2 * u3);
      S.R[0] = 1. - 2. * (qy * qy + qz * qz); S.R[1] = 2. * (qx * qy + qz * qw); S.R[2] = 2. * (qx * qz - qy * qw);
      S.R[3] = 2. * (qx * qy - qz * qw); S.R[4] = 1. - 2. * (qx * qx + qz * qz); S.R[5] = 2. * (qy * qz + qx * qw);
      S.R[6] = 2. * (qx * qz + qy * qw); S.R[7] = 2. * (qy * qz - qx * qw); S.R[8] = 1. - 2. * (qx * qx + qy * qy);
    }
    // a direction, a surface point along it, an offset along the normal
    const double zz = 2. * urand(seed, i, d++) - 1., ph = pi2 * urand(seed, i, d++);
    const double rr = sqrt(fmax(0., 1. - zz * zz));
    const double u[3] = {rr * cos(ph), rr * sin(ph), zz};
    const double off = 6. * urand(seed, i, d++) - 3.;
    double p[3];
    if (S.sphere) {
      for (int k = 0; k < 3; ++k) p[k] = S.c[k] + (S.s[0] + off) * u[k];
    } else {
      double g = 0.;
      for (int k = 0; k < 3; ++k) g += u[k] * u[k] / (S.s[k] * S.s[k]);
      double q[3], nq[3], nn = 0.;
      for (int k = 0; k < 3; ++k) {
        q[k] = u[k] / sqrt(g);
        nq[k] = q[k] / (S.s[k] * S.s[k]);
        nn += nq[k] * nq[k];
      }
      nn = sqrt(nn);
      double pb[3];
      for (int k = 0; k < 3; ++k) pb[k] = q[k] + off * nq[k] / nn;
      for (int k = 0; k < 3; ++k) p[k] = S.c[k] + S.R[k] * pb[0] + S.R[k + 3] * pb[1] + S.R[k + 6] * pb[2];
    }
    for (int k = 0; k < 3; ++k) x[k] = rint(p[k]);
    double foot[3];
    const double phi0 = sdist(S, x, foot);
    if (fabs(phi0) > 3.) continue;
    double k1, k2;
    if (S.sphere) {
      k1 = k2 = 1. / S.s[0];
    } else {
      ellipsoid_principal(S, foot, k1, k2);
    }
    // the level set through x: -(k1/(1+k1 phi) + k2/(1+k2 phi)), reference sign
    const double f1 = 1. + k1 * phi0, f2 = 1. + k2 * phi0;
    if (fmin(1. + k1 * (phi0 - 2.), 1. + k2 * (phi0 - 2.)) < 0.5) continue;
    kana = -(k1 / f1 + k2 / f2);
    if (fabs(kana) > 2. / 3.) continue;
    int q = 0;
    for (int dk = -1; dk <= 1; ++dk)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          const double pf[3] = {x[0] + 0.25 * di, x[1] + 0.25 * dj, x[2] + 0.25 * dk};
          ff[q++] = sdist(S, pf, nullptr);
        }
    lab = lsq_curv(ff, 0.25);
    if (fabs(lab - kana) > 0.02) continue;
    break;
  }
  double fc[27];
  int q = 0;
  for (int dk = -1; dk <= 1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        const double pc[3] = {x[0] + di, x[1] + dj, x[2] + dk};
        fc[q++] = sdist(S, pc, nullptr);
      }
  double fd[27];
  for (int k = 0; k < 27; ++k) fd[k] = fc[k] - fc[13];
  mlp_features(fd, X + i * kIn);
  const double plain = lsq_curv(fc, 1.);
  label[i] = (float)(lab - plain);  // the correction the network learns
  // the loss weight: errors relative to the curvature, so well-resolved
  // interfaces (small kappa dx, where the stencil is already accurate)
  // count as much as the under-resolved ones
  const double wr = 0.1 / (fabs(lab) + 0.02);
  weight[i] = (float)(wr * wr);
  extra[3 * i + 0] = (float)plain;
  extra[3 * i + 1] = (float)kana;
  extra[3 * i + 2] = (float)fmin(S.s[0], fmin(S.s[1], S.s[2]));
}


// ================================================ the network in the loop
// A gathered interface cell: task q of the batch, interior cell (i, j, k)

// The features of the recorded near-interface cells (k_curvature records
// the computed cells with |phi| <= 4dz, the cells re_curvature and the
// jumps read) into X, one thread per cell; cells beyond cap keep the plain
// curvature.
template <typename T>
__global__ void __launch_bounds__(256) k_mlp_features(Params p, const __grid_constant__ LsBatch B,
                                                      const MlpCell* __restrict__ rec, const int* __restrict__ count,
                                                      int cap, float* __restrict__ X) {
  const int n = min(*count, cap);
  const float rdz = (float)(1. / p.dz);
  const long long sy = p.nLx, sz = (long long)p.nLx * p.nLy;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const MlpCell r = rec[s];
    const T* __restrict__ phi = cT<T>(B.t[r.q].phi0);
    const long long cl = idxL(p, r.i, r.j, r.k);
    float f[27];
    int m = 0;
    for (int dk = -1; dk <= 1; ++dk)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) f[m++] = (float)phi[cl + di + dj * sy + dk * sz];
    const float pc = f[13];
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = (f[q] - pc) * rdz;
    float o[kIn];
    mlp_features(f, o);
    float4* dst = reinterpret_cast<float4*>(X + (long long)s * kIn);
#pragma unroll
    for (int q = 0; q < kIn / 4; ++q) dst[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
  }
}

// the learned curvature kappa_plain + y/dx where it passes the checks, the
// plain one otherwise (a correction |y| > tol, or a curvature radius below 3
// cells, |kappa_plain| dx > 2/3), written straight from the last layer's
// epilogue of the gathered cells' tiles
template <typename T>
struct ApplyOut {
  const Params& p;
  const LsBatch& B;
  const MlpCell* __restrict__ rec;
  double tol;
  unsigned long long ev, fb;
  MlpCell r;  // this thread's cell of the current tile and its stencil curvature
  double kp;
  __device__ void begin(long long s, bool live) {
    if (!live) return;
    r = rec[s];
    kp = (double)mT<T>(B.t[r.q].out)[idxC(p, r.i, r.j, r.k)];
  }
  __device__ void operator()(long long, float y) {
    T* out = mT<T>(B.t[r.q].out);
    const double dz = p.dz;
    double km = kp + (double)y / dz;
    ++ev;
    if (fabs(kp) * dz > 2. / 3. || fabs(km - kp) * dz > tol) {
      ++fb;
      return;
    }
    const double maxk = 1. / dz;  // the clamps of interface.f90:104-111
    if (km < -maxk) km = -maxk;
    else if (km > maxk) km = maxk;
    else if (fabs(km) < 1e-9) km = 0.;
    putC(p, out, r.i, r.j, r.k, (T)km);
  }
};

// the network over the first min(*count, cap) gathered cells and the
// per-cell choice; stats[0] += evaluated, stats[1] += fallbacks
template <typename T>
__global__ void __launch_bounds__(128, 2) k_mlp_curv(Net net, const float* __restrict__ X,
                                                     const int* __restrict__ count, int cap, Params p,
                                                     const __grid_constant__ LsBatch B,
                                                     const MlpCell* __restrict__ rec, double tol,
                                                     unsigned long long* __restrict__ stats, int* __restrict__ err) {
  const long long n = min(*count, cap);
  ApplyOut<T> o{p, B, rec, tol, 0ull, 0ull, MlpCell{0, 0, 0, 0}, 0.};
  infer_tiles(net, X, n, o, err);
  unsigned long long ev = o.ev, fb = o.fb;
  for (int d = 16; d > 0; d >>= 1) {
    ev += __shfl_down_sync(0xffffffffu, ev, d);
    fb += __shfl_down_sync(0xffffffffu, fb, d);
  }
  if ((threadIdx.x & 31) == 0 && ev) {
    atomicAdd(stats, ev);
    atomicAdd(stats + 1, fb);
  }
}
}  // namespace
}  // namespace icls

struct icls_mlp {
  float *theta = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *w2t = nullptr, *w3t = nullptr;
  float* zbuf = nullptr;     // pre-activations of one batch
  long long zcap = 0;        // samples zbuf holds
  float* loss = nullptr;     // per-epoch loss sums
  int nloss = 0;
  int* err = nullptr;
  float* X = nullptr;          // training inputs [n][32]
  float *label = nullptr, *weight = nullptr, *extra = nullptr;
  long long n_train = 0;
  float* Xh = nullptr;         // held-out set
  float *labelh = nullptr, *weighth = nullptr, *extrah = nullptr, *yh = nullptr;
  long long n_hold = 0;
  long long step = 0;
  cudaStream_t s = nullptr;
};

namespace {
using namespace icls;

Net net_of(const icls_mlp* m) { return Net{m->theta, m->w1, m->w2, m->w3, m->w2t, m->w3t}; }

unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int sync_err(icls_mlp* m) {
  int h = 0;
  if (cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->s) != cudaSuccess) return ICLS_E_CUDA;
  if (cudaStreamSynchronize(m->s) != cudaSuccess) return ICLS_E_CUDA;
  if (cudaGetLastError() != cudaSuccess) return ICLS_E_CUDA;
  return h ? ICLS_E_CUDA : ICLS_OK;
}

int ensure_zbuf(icls_mlp* m, long long n) {
  if (n <= m->zcap) return ICLS_OK;
  if (m->zbuf) cudaFree(m->zbuf);
  m->zbuf = nullptr;
  if (cudaMalloc(&m->zbuf, sizeof(float) * (size_t)n * (kH1 + kH2 + kH3)) != cudaSuccess) return ICLS_E_NOMEM;
  m->zcap = n;
  return ICLS_OK;
}

void refresh_copies(icls_mlp* m) {
  k_mlp_copies<<<(kParams + 255) / 256, 256, 0, m->s>>>(m->theta, m->w1, m->w2, m->w3, m->w2t, m->w3t);
}

}  // namespace

namespace icls {
// get_curvature's output (the batch tasks' out buffers, computed by
// launch_curvature with collect set, which also recorded the cells)
// replaced by the network near the interface
int launch_mlp_curvature(Ctx& c, const LsBatch& b) {
  if (b.n == 0) return ICLS_OK;
  if (!c.net) return ICLS_E_STATE;
  Scope sc_(c.prof, c.s, "mlp_curvature", 2);
  if (c.P.f32)
    k_mlp_features<float><<<4 * 148, 256, 0, c.s>>>(c.P, b, (const MlpCell*)c.mlp_rec, c.mlp_count, c.mlp_cap,
                                                    c.mlp_X);
  else
    k_mlp_features<double><<<4 * 148, 256, 0, c.s>>>(c.P, b, (const MlpCell*)c.mlp_rec, c.mlp_count, c.mlp_cap,
                                                     c.mlp_X);
  const int grid = std::min((c.mlp_cap + kRows - 1) / kRows, 2 * 148);
  const double tol = c.cfg.mlp_fallback_tol;
  if (c.P.f32)
    k_mlp_curv<float><<<grid, 128, SB_INFER, c.s>>>(net_of(c.net), c.mlp_X, c.mlp_count, c.mlp_cap, c.P, b,
                                                    (const MlpCell*)c.mlp_rec, tol, c.mlp_stats, c.net->err);
  else
    k_mlp_curv<double><<<grid, 128, SB_INFER, c.s>>>(net_of(c.net), c.mlp_X, c.mlp_count, c.mlp_cap, c.P, b,
                                                     (const MlpCell*)c.mlp_rec, tol, c.mlp_stats, c.net->err);
  return ICLS_OK;
}

// the unit-spacing pseudo-inverse the features and the labels use (once per
// process and device-wide)
int mlp_constants() {
  static unsigned set = 0;  // devices the constants are on
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (set & (1u << (dev & 31))) return 0;
  double pu[270];
  float puf[270];
  pseudo_inverse(1., 1., 1., pu);
  for (int q = 0; q < 270; ++q) puf[q] = (float)pu[q];
  if (cudaMemcpyToSymbol(cPu, pu, sizeof(pu)) != cudaSuccess) return 1;
  if (cudaMemcpyToSymbol(cPuf, puf, sizeof(puf)) != cudaSuccess) return 1;
  set |= 1u << (dev & 31);
  return 0;
}

// device buffers of the context's gathered cells (16-byte cell records)
int mlp_buffers(Ctx& c, int cap) {
  if (mlp_constants()) return ICLS_E_CUDA;
  if (cudaMalloc(&c.mlp_X, (size_t)cap * kIn * 4) != cudaSuccess) return ICLS_E_NOMEM;
  if (cudaMalloc(&c.mlp_rec, (size_t)cap * sizeof(MlpCell)) != cudaSuccess) return ICLS_E_NOMEM;
  if (cudaMalloc(&c.mlp_count, sizeof(int)) != cudaSuccess) return ICLS_E_NOMEM;
  if (cudaMalloc(&c.mlp_stats, 2 * sizeof(unsigned long long)) != cudaSuccess) return ICLS_E_NOMEM;
  cudaMemset(c.mlp_stats, 0, 2 * sizeof(unsigned long long));
  c.mlp_cap = cap;
  return cudaFuncSetAttribute(k_mlp_curv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, SB_INFER) ==
                     cudaSuccess &&
                 cudaFuncSetAttribute(k_mlp_curv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, SB_INFER) ==
                     cudaSuccess
             ? ICLS_OK
             : ICLS_E_CUDA;
}
}  // namespace icls

extern "C" int icls_mlp_create(icls_mlp** out, unsigned long long seed) {
  if (!out) return ICLS_E_ARG;
  *out = nullptr;
  icls_mlp* m = new (std::nothrow) icls_mlp();
  if (!m) return ICLS_E_NOMEM;
  bool ok = cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) == cudaSuccess;
  for (float** f : {&m->theta, &m->grad, &m->m1, &m->m2}) ok = ok && cudaMalloc(f, sizeof(float) * kParams) == cudaSuccess;
  ok = ok && cudaMalloc(&m->w1, 2 * kH1 * kIn2) == cudaSuccess && cudaMalloc(&m->w2, 2 * kH2 * kH1) == cudaSuccess &&
       cudaMalloc(&m->w3, 2 * kH3 * kH2) == cudaSuccess && cudaMalloc(&m->w2t, 2 * kH2 * kH1) == cudaSuccess &&
       cudaMalloc(&m->w3t, 2 * kH3 * kH2) == cudaSuccess && cudaMalloc(&m->err, sizeof(int)) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(icls::k_mlp_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, icls::SB_TRAIN) ==
                 cudaSuccess &&
       cudaFuncSetAttribute(icls::k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, icls::SB_INFER) ==
           cudaSuccess;
  if (!ok) {
    icls_mlp_destroy(m);
    return ICLS_E_NOMEM;
  }
  // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases; the
  // padding inputs 27..31 of W1 stay zero
  std::vector<float> th(kParams, 0.f);
  unsigned long long st = seed;
  auto unif = [&](float a) {
    st = mix64(st);
    return (float)((double)(st >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0) * a;
  };
  for (int r = 0; r < kH1; ++r)
    for (int c = 0; c < 27; ++c) th[oW1 + r * kIn + c] = unif(1.f / sqrtf(27.f));
  for (int q = 0; q < kH2 * kH1; ++q) th[oW2 + q] = unif(1.f / sqrtf((float)kH1));
  for (int q = 0; q < kH3 * kH2; ++q) th[oW3 + q] = unif(1.f / sqrtf((float)kH2));
  for (int q = 0; q < kH3; ++q) th[oW4 + q] = unif(1.f / sqrtf((float)kH3));
  cudaMemcpyAsync(m->theta, th.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, m->s);
  for (float* f : {m->grad, m->m1, m->m2}) cudaMemsetAsync(f, 0, sizeof(float) * kParams, m->s);
  cudaMemsetAsync(m->err, 0, sizeof(int), m->s);
  refresh_copies(m);
  if (cudaStreamSynchronize(m->s) != cudaSuccess) {
    icls_mlp_destroy(m);
    return ICLS_E_CUDA;
  }
  *out = m;
  return ICLS_OK;
}

extern "C" int icls_mlp_destroy(icls_mlp* m) {
  if (!m) return ICLS_E_ARG;
  if (m->s) cudaStreamSynchronize(m->s);
  for (void* p : {(void*)m->theta, (void*)m->grad, (void*)m->m1, (void*)m->m2, (void*)m->w1, (void*)m->w2,
                  (void*)m->w3, (void*)m->w2t, (void*)m->w3t, (void*)m->zbuf, (void*)m->loss, (void*)m->err,
                  (void*)m->X, (void*)m->label, (void*)m->weight, (void*)m->extra, (void*)m->Xh, (void*)m->labelh,
                  (void*)m->weighth, (void*)m->extrah, (void*)m->yh})
    if (p) cudaFree(p);
  if (m->s) cudaStreamDestroy(m->s);
  delete m;
  return ICLS_OK;
}

// n_train a power of two (the epoch shuffle is an affine map mod n_train)
extern "C" int icls_mlp_make_data(icls_mlp* m, unsigned long long seed, long long n_train, long long n_hold) {
  if (!m || n_train < 128 || (n_train & (n_train - 1)) || n_hold < 1) return ICLS_E_ARG;
  if (icls::mlp_constants()) return ICLS_E_CUDA;
  for (void* p : {(void*)m->X, (void*)m->label, (void*)m->weight, (void*)m->extra, (void*)m->Xh, (void*)m->labelh,
                  (void*)m->weighth, (void*)m->extrah, (void*)m->yh})
    if (p) cudaFree(p);
  m->X = m->Xh = nullptr;
  m->label = m->weight = m->extra = m->labelh = m->weighth = m->extrah = m->yh = nullptr;
  bool ok = cudaMalloc(&m->X, 4 * (size_t)n_train * kIn) == cudaSuccess &&
            cudaMalloc(&m->label, 4 * (size_t)n_train) == cudaSuccess &&
            cudaMalloc(&m->weight, 4 * (size_t)n_train) == cudaSuccess &&
            cudaMalloc(&m->weighth, 4 * (size_t)n_hold) == cudaSuccess &&
            cudaMalloc(&m->extra, 12 * (size_t)n_train) == cudaSuccess &&
            cudaMalloc(&m->Xh, 4 * (size_t)n_hold * kIn) == cudaSuccess &&
            cudaMalloc(&m->labelh, 4 * (size_t)n_hold) == cudaSuccess &&
            cudaMalloc(&m->extrah, 12 * (size_t)n_hold) == cudaSuccess &&
            cudaMalloc(&m->yh, 4 * (size_t)n_hold) == cudaSuccess;
  if (!ok) return ICLS_E_NOMEM;
  m->n_train = n_train;
  m->n_hold = n_hold;
  icls::k_mlp_gen<<<(unsigned)((n_train + 127) / 128), 128, 0, m->s>>>(seed, n_train, m->X, m->label, m->weight,
                                                                       m->extra);
  icls::k_mlp_gen<<<(unsigned)((n_hold + 127) / 128), 128, 0, m->s>>>(mix64(seed ^ 0x5bd1e995ull), n_hold, m->Xh,
                                                                      m->labelh, m->weighth, m->extrah);
  return sync_err(m);
}

// epochs over the training set in batches of `batch` (a multiple of 128
// dividing n_train), Adam with a step size decaying from lr to lr_final
// along a half cosine; loss_out[e] = mean squared error of epoch e
// (kappa*dx units), if given
extern "C" int icls_mlp_train(icls_mlp* m, int epochs, int batch, double lr, double lr_final,
                              unsigned long long seed, double* loss_out) {
  if (!m || !m->X || epochs < 1 || batch < 128 || batch % 128 || m->n_train % batch) return ICLS_E_ARG;
  int rc = ensure_zbuf(m, batch);
  if (rc) return rc;
  if (m->nloss < epochs) {
    if (m->loss) cudaFree(m->loss);
    if (cudaMalloc(&m->loss, sizeof(float) * epochs) != cudaSuccess) return ICLS_E_NOMEM;
    m->nloss = epochs;
  }
  cudaMemsetAsync(m->loss, 0, sizeof(float) * epochs, m->s);
  const Net net = net_of(m);
  const long long steps = m->n_train / batch;
  const long long total = steps * epochs;
  long long done = 0;
  const float scale = 2.f / (float)batch;
  for (int e = 0; e < epochs; ++e) {
    const unsigned long long pa = mix64(seed + 2 * (unsigned long long)e) | 1ull;
    const unsigned long long pb = mix64(seed + 2 * (unsigned long long)e + 1);
    for (long long st = 0; st < steps; ++st) {
      icls::k_mlp_train_tile<<<batch / 128, 128, icls::SB_TRAIN, m->s>>>(net, m->X, m->label, m->weight, m->n_train,
                                                                          st * batch, pa, pb, scale, m->zbuf,
                                                                          m->grad, m->loss + e, m->err);
      ++m->step;
      const double lr_t = lr_final + 0.5 * (lr - lr_final) * (1. + std::cos(3.141592653589793 * (double)done / (double)total));
      ++done;
      const float bc1 = 1.f - powf(0.9f, (float)m->step), bc2 = 1.f - powf(0.999f, (float)m->step);
      icls::k_mlp_adam<<<(kParams + 255) / 256, 256, 0, m->s>>>(m->theta, m->grad, m->m1, m->m2, (float)lr_t, bc1,
                                                                 bc2, m->w1, m->w2, m->w3, m->w2t, m->w3t);
    }
  }
  rc = sync_err(m);
  if (rc) return rc;
  if (loss_out) {
    std::vector<float> l(epochs);
    cudaMemcpy(l.data(), m->loss, sizeof(float) * epochs, cudaMemcpyDeviceToHost);
    for (int e = 0; e < epochs; ++e) loss_out[e] = l[e] / (double)m->n_train;
  }
  return ICLS_OK;
}

// y[0..n) = network(X[0..n)) on device arrays (X FP32 [n][32])
extern "C" int icls_mlp_infer(icls_mlp* m, const void* X, float* y, long long n, void* stream) {
  if (!m || !X || !y || n < 1 || (reinterpret_cast<uintptr_t>(X) & 15)) return ICLS_E_ARG;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m->s;
  const long long tiles = (n + 127) / 128;
  const int grid = (int)std::min<long long>(tiles, 2 * 148);
  icls::k_mlp_infer<<<grid, 128, icls::SB_INFER, s>>>(net_of(m), static_cast<const float*>(X), n, y, m->err);
  if (stream) return cudaGetLastError() == cudaSuccess ? ICLS_OK : ICLS_E_CUDA;
  return sync_err(m);
}

// statistics of the held-out set, kappa*dx units: stats[0..3] = rms of
// (mlp - label), (mlp - analytic), (plain - analytic), (label - analytic);
// stats[4..5] = max |mlp - analytic|, max |plain - analytic|; stats[6] =
// rms |analytic|; stats[7] = samples
extern "C" int icls_mlp_eval(icls_mlp* m, double* stats) {
  if (!m || !m->Xh || !stats) return ICLS_E_ARG;
  int rc = icls_mlp_infer(m, m->Xh, m->yh, m->n_hold, nullptr);
  if (rc) return rc;
  const size_t n = (size_t)m->n_hold;
  std::vector<float> y(n), lab(n), ex(3 * n);
  cudaMemcpy(y.data(), m->yh, 4 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(lab.data(), m->labelh, 4 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(ex.data(), m->extrah, 12 * n, cudaMemcpyDeviceToHost);
  double s[8] = {0, 0, 0, 0, 0, 0, 0, (double)n};
  for (size_t i = 0; i < n; ++i) {
    const double ka = ex[3 * i + 1], kp = ex[3 * i + 0];
    const double km = kp + y[i], kl = kp + lab[i];  // learned and refined-grid curvature
    s[0] += (km - kl) * (km - kl);
    s[1] += (km - ka) * (km - ka);
    s[2] += (kp - ka) * (kp - ka);
    s[3] += (kl - ka) * (kl - ka);
    s[4] = std::max(s[4], std::fabs(km - ka));
    s[5] = std::max(s[5], std::fabs(kp - ka));
    s[6] += ka * ka;
  }
  for (int q : {0, 1, 2, 3, 6}) s[q] = std::sqrt(s[q] / (double)n);
  for (int q = 0; q < 8; ++q) stats[q] = s[q];
  return ICLS_OK;
}

// the FP32 parameters (29057 floats in the layout of k_mlp.cu) to or from host
extern "C" int icls_mlp_params(icls_mlp* m, float* host, int get) {
  if (!m || !host) return ICLS_E_ARG;
  if (get) {
    if (cudaMemcpy(host, m->theta, sizeof(float) * kParams, cudaMemcpyDeviceToHost) != cudaSuccess) return ICLS_E_CUDA;
    return ICLS_OK;
  }
  if (cudaMemcpy(m->theta, host, sizeof(float) * kParams, cudaMemcpyHostToDevice) != cudaSuccess) return ICLS_E_CUDA;
  refresh_copies(m);
  return sync_err(m);
}

// the gradient of the summed squared error x scale over samples 0..n-1 of X
// (device FP32 [n][32], labels device FP32), n a power of two >= 128, into
// host grad[29057]; loss = sum of squared errors
extern "C" int icls_mlp_grad(icls_mlp* m, const void* X, const float* label, long long n, float scale, float* grad,
                             double* loss) {
  if (!m || !X || !label || !grad || n < 128 || (n & (n - 1))) return ICLS_E_ARG;
  int rc = ensure_zbuf(m, n);
  if (rc) return rc;
  if (m->nloss < 1) {
    if (cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess) return ICLS_E_NOMEM;
    m->nloss = 1;
  }
  cudaMemsetAsync(m->loss, 0, sizeof(float), m->s);
  cudaMemsetAsync(m->grad, 0, sizeof(float) * kParams, m->s);
  icls::k_mlp_train_tile<<<(unsigned)(n / 128), 128, icls::SB_TRAIN, m->s>>>(
      net_of(m), static_cast<const float*>(X), label, nullptr, n, 0, 1ull, 0ull, scale, m->zbuf, m->grad, m->loss,
      m->err);
  rc = sync_err(m);
  if (rc) return rc;
  cudaMemcpy(grad, m->grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost);
  float l = 0.f;
  cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
  if (loss) *loss = l;
  cudaMemset(m->grad, 0, sizeof(float) * kParams);
  return ICLS_OK;
}

extern "C" int icls_tc_gemm_bf16(const void* a, const void* b, float* d, int n, int k, void* stream) {
  if (!a || !b || !d) return ICLS_E_ARG;
  if (n < 16 || n > 128 || n % 16 || k < 16 || k > 128 || k % 16) return ICLS_E_ARG;
  int* err = nullptr;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return ICLS_E_NOMEM;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(err, 0, sizeof(int), s);
  const int smem = 2 * 128 * 128 * 2;
  cudaFuncSetAttribute(icls::k_tc_gemm_check, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  icls::k_tc_gemm_check<<<1, 128, smem, s>>>(static_cast<const __nv_bfloat16*>(a), static_cast<const __nv_bfloat16*>(b),
                                          d, n, k, err);
  int h = 0;
  cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(err);
  if (e != cudaSuccess) return ICLS_E_CUDA;
  return h ? ICLS_E_CUDA : ICLS_OK;
}
