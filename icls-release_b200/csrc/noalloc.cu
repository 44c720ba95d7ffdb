// noalloc.cu — the divergence check of chkdiv (chkdiv.f90:10-90) for callers
// that cannot allocate device memory.
//
// Who needs it: a host code that has already claimed the device memory it
// is allowed to use — for instance a Fortran driver that sizes all of its
// fields at start-up through its own pool and treats any later allocation
// as an error, or a diagnostics hook run between time steps of such a
// simulation, where an out-of-memory failure inside a check is not
// acceptable.  Such a caller owns u, v, w and the result buffer and cannot
// let the library cudaMalloc the per-block partial sums that
// icls_chkdiv keeps in its context.
//
// Here those partials live in g_scratch, a file-scope __device__ array of
// fixed size: every GPU that loads the library holds it (about 28 KB) until
// the process exits.  Host code may not use the symbol g_scratch as a device
// address; the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it.  That first
// call should therefore be made before any stream capture.  Every call
// shares the array and leaves its contents behind: each call rewrites all
// partial slots before reading them, so nothing needs clearing, but calls
// that overlap on the GPU (different streams, no ordering) race on it.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>

#include "../../include/icls_gpu.h"

namespace {

constexpr int kBlocks = 1184;   // 8 blocks per SM on 148 SMs
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// [sums | maxima | locations] of every block; locations are cell indices
// stored exactly as doubles (< 2^31)
static __device__ __align__(256) double g_scratch[3 * kBlocks];

void* g_addr[kMaxDevices] = {nullptr};
std::mutex g_mu;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// per-block sum of div and max|div| with its first column-major location,
// the same partition and order as the context path
__global__ void __launch_bounds__(kThreads) k_div_partials(const double* __restrict__ u,
                                                           const double* __restrict__ v,
                                                           const double* __restrict__ w, int imax, int jmax,
                                                           int kmax, double dxi, double dyi, double dzi,
                                                           double* __restrict__ scratch) {
  const int nCx = imax + 2, nCy = jmax + 2;
  const long long sz = (long long)nCx * nCy;
  // 64-bit counter and stride: with nI up to 2^31-1 the last q + stride
  // passes INT_MAX and would wrap a 32-bit index to a negative cell
  const long long nI = (long long)imax * jmax * kmax;
  const long long stride = (long long)gridDim.x * kThreads;
  double s = 0., m = 0.;
  long long loc = -1;
  for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < nI; q += stride) {
    const int i = (int)(q % imax) + 1;
    const long long r = q / imax;
    const int j = (int)(r % jmax) + 1;
    const long long k = r / jmax + 1;
    const long long c = (long long)i + (long long)nCx * ((long long)j + (long long)nCy * k);
    double div = ((w[c] - w[c - sz]) * dzi + (v[c] - v[c - nCx]) * dyi) + (u[c] - u[c - 1]) * dxi;
    s += div;
    div = fabs(div);
    if (div > m) {
      m = div;
      loc = q;
    }
  }
  __shared__ double red[kThreads / 32];
  __shared__ double sm[kThreads];
  __shared__ long long sl[kThreads];
  double ws = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ws;
  sm[threadIdx.x] = m;
  sl[threadIdx.x] = loc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double b = (threadIdx.x < kThreads / 32) ? red[threadIdx.x] : 0.;
    b = warp_sum(b);
    if (threadIdx.x == 0) {
      double bm = 0.;
      long long bl = -1;
      for (int t = 0; t < kThreads; ++t)
        if (sm[t] > bm || (sm[t] == bm && sm[t] > 0. && sl[t] < bl)) {
          bm = sm[t];
          bl = sl[t];
        }
      scratch[blockIdx.x] = b;
      scratch[kBlocks + blockIdx.x] = bm;
      scratch[2 * kBlocks + blockIdx.x] = (double)bl;
    }
  }
}

// combine the partials in block order; result = [divtot, divmax, i, j, k]
__global__ void k_div_final(const double* __restrict__ scratch, int imax, int jmax, double* __restrict__ result) {
  if (threadIdx.x != 0) return;
  double s = 0., m = 0., l = -1.;
  for (int b = 0; b < kBlocks; ++b) {
    s += scratch[b];
    const double pm = scratch[kBlocks + b], pl = scratch[2 * kBlocks + b];
    if (pm > m || (pm == m && pm > 0. && pl < l)) {
      m = pm;
      l = pl;
    }
  }
  result[0] = s;
  result[1] = m;
  if (l < 0.) {
    result[2] = result[3] = result[4] = 0.;
  } else {
    const long long q = (long long)l;
    result[2] = (double)(q % imax + 1);
    result[3] = (double)((q / imax) % jmax + 1);
    result[4] = (double)(q / ((long long)imax * jmax) + 1);
  }
}

// device address of g_scratch on the current device, looked up once
int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ICLS_E_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return ICLS_E_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return ICLS_E_CUDA;
    g_addr[dev] = p;
  }
  *out = static_cast<double*>(g_addr[dev]);
  return ICLS_OK;
}

}  // namespace

extern "C" int icls_chkdiv_noalloc(const double* u, const double* v, const double* w, int imax, int jmax, int kmax,
                                   double dxi, double dyi, double dzi, double* result, void* stream) {
  if (!u || !v || !w || !result) return ICLS_E_ARG;
  if (imax < 1 || jmax < 1 || kmax < 1) return ICLS_E_ARG;
  // locations travel as doubles and the result's k is computed from them:
  // the limit keeps every cell index exact and far inside 64-bit arithmetic
  if ((long long)imax * jmax * kmax > (long long)ICLS_NOALLOC_MAX_CELLS) return ICLS_E_SIZE;
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_div_partials<<<kBlocks, kThreads, 0, s>>>(u, v, w, imax, jmax, kmax, dxi, dyi, dzi, scratch);
  k_div_final<<<1, 32, 0, s>>>(scratch, imax, jmax, result);
  return cudaGetLastError() == cudaSuccess ? ICLS_OK : ICLS_E_CUDA;
}
