// umma.cuh — one CTA's 128 x N BF16 tensor-core tile on sm_100a (tcgen05).
//
// D[128 x N] (FP32, in tensor memory) = A[128 x K] * B[N x K]^T, A and B
// BF16 in shared memory in the canonical K-major layout without swizzle:
// the K extent is cut into 8-element (16-byte) chunks; chunk c of row r
// sits at  c * (rows * 16) + r * 16  bytes, so a "core matrix" (8 rows x
// 16 bytes) is 128 contiguous bytes, 8-row groups are 128 bytes apart (the
// descriptor's stride byte offset) and consecutive K chunks rows*16 bytes
// apart (its leading byte offset).  One elected thread issues K/16 MMAs of
// shape 128 x N x 16 and commits them to an mbarrier; the CTA waits on the
// barrier with an iteration limit.  Thread t of the 128-thread CTA then
// owns row t of D (tensor-memory lane t).
//
// Descriptor encodings follow the PTX ISA's tcgen05 shared-memory and
// instruction descriptors (field positions as documented there and in the
// CUTLASS sm100 headers): version 1, no swizzle; kind::f16 with BF16 A/B,
// FP32 D, both operands K-major, N>>3 at bit 17, M>>4 at bit 24.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace icls {
namespace umma {

constexpr int kRows = 128;                // M of every tile
constexpr long long kWaitLimit = 1 << 26; // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(const void* base, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  const uint64_t a = (smem_u32(base) >> 4) & 0x3FFFu;
  const uint64_t l = (lbo_bytes >> 4) & 0x3FFFu;
  const uint64_t s = (sbo_bytes >> 4) & 0x3FFFu;
  return a | (l << 16) | (s << 32) | (1ull << 46);  // layout type 0 (no swizzle) in bits 61..63
}

// instruction descriptor: kind::f16, A = B = BF16, D = FP32, K-major, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4)            // D format F32
         | (1u << 7)          // A format BF16
         | (1u << 10)         // B format BF16
         | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

// byte offset of element (r, k) in a K-major no-swizzle tile with `rows` rows
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int rows) {
  return (uint32_t)((k >> 3) * rows * 16 + r * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// wait for the barrier's phase `parity` to complete; false after the limit
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// tensor memory: one warp allocates `cols` columns (power of two >= 32) and
// writes the base address to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols));
}

// D (+)= A * B^T for one 128 x n x 16 step, issued by the calling thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 8 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld8(uint32_t addr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[q]);
}

// 32 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// The tile product of the CTA: a (128 x k) and b (n x k) in the layout
// above, k a multiple of 16, n a multiple of 16 up to 256, result in the
// tensor-memory columns d_tmem .. d_tmem+n-1.  All 128 threads call it after
// the operands are in shared memory; returns false if the wait gave up.
__device__ __forceinline__ bool tile_gemm(const void* a, const void* b, int n, int k, uint32_t d_tmem, uint64_t* bar,
                                          uint32_t& phase) {
  fence_async_smem();  // the operands' generic-proxy stores before the tensor core reads them
  fence_before();      // earlier tensor-memory reads before the columns are overwritten
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after();
    const uint32_t id = idesc_bf16(n);
    for (int s = 0; s < k / 16; ++s) {
      const char* as = static_cast<const char*>(a) + (size_t)s * 2 * kRows * 16;
      const char* bs = static_cast<const char*>(b) + (size_t)s * 2 * n * 16;
      mma_bf16(d_tmem, smem_desc(as, kRows * 16, 128), smem_desc(bs, (uint32_t)n * 16, 128), id, s > 0 ? 1u : 0u);
    }
    mma_commit(bar);
  }
  const bool ok = mbar_wait(bar, phase);
  phase ^= 1u;
  fence_after();
  return ok;
}

}  // namespace umma
}  // namespace icls
