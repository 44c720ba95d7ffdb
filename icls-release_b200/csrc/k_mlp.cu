// k_mlp.cu — the learned interface curvature: a 27-128-128-64-1 SiLU MLP
// on tcgen05 tensor-core tiles (BF16 operands, FP32 accumulation in tensor
// memory).  Compiled without -fmad=false: this is not reference arithmetic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/icls_gpu.h"
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

}  // namespace
}  // namespace icls

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
