// k_ab2_tma.cu — the plain FP64 AB2 predictor (ab2.f90:21-138 with
// mom_main's RHS, mom.f90:13-301, and the wall rows of bounduvw(dudt,..),
// bound.f90:36-75) fed by the Tensor Memory Accelerator.
//
// Opt-in (ICLS_AB2=tma): at 256^3 it measured 1.68 ms against the
// cp.async-ring kernel's 1.37 ms, so the ring stays the default; 16 compute
// warps per SM (the most the 128-register budget of the FP64 stencil
// arithmetic allows with one CTA) hide less latency than the ring's two
// CTAs, each of which overlaps the other's waits.
//
// The arithmetic per cell is the one of k_ab2 in ab2.cuh (the same rhs_u/v/w
// and ab2_update_v templates, compiled with -fmad=false), so the result is
// bit-identical to it.  What changes is how the 18 input fields reach the
// SM.  A persistent CTA (one per SM, 16 warps) walks work items = (32 x 16
// column tile, chunk of z rows).  Thread 0 issues, per row, 3-D TMA box
// loads of every field into two shared-memory rings, completed on
// mbarriers: the stencil fields two rows ahead of the row being computed,
// the pointwise fields one row ahead.  Each warp waits for the rows it
// needs and releases a slot with one arrive; no thread issues a global load
// and no block-wide barrier runs inside the loop.
//
//   stencil ring (SR = 4 rows):   u, v, w, miu, pnew, pold — shape C,
//                                 box 34 x 18 at (i0-1, j0-1, k)
//   pointwise ring (PR = 2 rows): p_x, p_y, p_z and their old values —
//                                 shape C, box 34 x 16 at (i0-1, j0, k);
//                                 rho_u, rho_v, rho_w, duold, dvold, dwold —
//                                 shape I, box 32 x 16 at (i0, j0, k)
//
// The tensor maps cover this GPU's own arrays only, and each load fills
// only the issuing CTA's shared memory.  Every box starts at an even x index (32 * tile, element
// size 8 B), every row pitch is a multiple of 16 B (imax even), and each
// shared-memory box starts on a 128-byte boundary.  Every mbarrier wait has
// an iteration limit: on expiry the kernel sets DevScalars::wait_err, thread
// 0 lets its outstanding copies land (bounded again) and all threads
// return.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "ab2.cuh"
#include "ctx.h"

namespace icls {
namespace {

constexpr int TX = 32, TY = 16;                  // column tile
constexpr int SW = TX + 2, SH = TY + 2;          // stencil box 34 x 18
constexpr int SR = 4, PR = 2;                    // ring slots
constexpr int NW = TY;                           // warps: one tile row each
constexpr int kThreadsTma = 32 * NW;
constexpr int kStBytes = SW * SH * 8;            // 4896 B a stencil box delivers
constexpr int kStBox = 4992;                     // padded to 128 B
constexpr int kPgBox = SW * TY * 8;              // 4352 B (34 x 128)
constexpr int kPiBox = TX * TY * 8;              // 4096 B
constexpr int kStSlot = 6 * kStBox;              // 29952
constexpr int kPwSlot = 6 * kPgBox + 6 * kPiBox; // 50688
constexpr int kStTx = 6 * kStBytes;              // expect-tx bytes per stencil row
constexpr int kPwTx = kPwSlot;                   // per pointwise row
constexpr int kRowsPerItem = 32;
constexpr long long kSpin = 1 << 24;             // mbarrier polls before giving up
constexpr int kSmemTma = SR * kStSlot + PR * kPwSlot + 2 * (SR + PR) * 8 + 16 + 32;  // + flag, cursors
static_assert(kStBytes <= kStBox && kStBox % 128 == 0 && kPgBox % 128 == 0 && kPiBox % 128 == 0, "box layout");
static_assert(kSmemTma <= 232448, "shared memory of one CTA");

struct Ab2Maps {
  CUtensorMap st[6];  // u v w miu pnew pold
  CUtensorMap pg[6];  // px py pz pxold pyold pzold
  CUtensorMap pi[6];  // rho_u rho_v rho_w duold dvold dwold
};

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// wait for phase `parity` of the barrier; false after kSpin polls, or as
// soon as another warp of the CTA has raised *abort (checked every 64 polls)
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, const volatile int* abort) {
  for (long long it = 0; it < kSpin; ++it) {
    if ((it & 63) == 63 && abort && *abort) return false;
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void bar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// 3-D tiled TMA load of one box into this CTA's own shared memory
__device__ __forceinline__ void tma3(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

struct Item {
  int i0, j0, ka, kb;  // tile origin (interior indices) and rows
};
__device__ __forceinline__ Item item_of(const Params& p, int it, int ntx, int nty, int nch, int kc) {
  const int nt = ntx * nty;
  const int t = it % nt, ch = it / nt;
  Item r;
  r.i0 = 1 + TX * (t % ntx);
  r.j0 = 1 + TY * (t / ntx);
  r.ka = 1 + ch * kc;
  r.kb = (ch == nch - 1) ? p.kmax : r.ka + kc - 1;
  return r;
}

// The issuing side of one ring: the next row to load (item `it`, row kk)
// and the positions issued so far.  Stencil rows of an item run ka-1 ..
// kb+1, pointwise rows ka .. kb.
struct Cursor {
  int it, kk;
  long long n;
};

__global__ void __launch_bounds__(kThreadsTma, 1)
    k_ab2_tma(const __grid_constant__ Ab2Maps maps, Params p, const double* __restrict__ rho_avr_p,
              double* __restrict__ dudt, double* __restrict__ dvdt, double* __restrict__ dwdt,
              double* __restrict__ duold_out, double* __restrict__ dvold_out, double* __restrict__ dwold_out,
              DevScalars* __restrict__ dsc, int ntx, int nty, int nch, int kc) {
  extern __shared__ __align__(128) unsigned char tsm[];
  unsigned char* st_base = tsm;
  unsigned char* pw_base = tsm + SR * kStSlot;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tsm + SR * kStSlot + PR * kPwSlot);
  uint64_t* st_full = bars;
  uint64_t* st_empty = bars + SR;
  uint64_t* pw_full = bars + 2 * SR;
  uint64_t* pw_empty = bars + 2 * SR + PR;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 2 * (SR + PR));
  // thread 0's issuing state, in shared memory to keep the compute
  // threads' registers free
  Cursor& cs = *reinterpret_cast<Cursor*>(tsm + SR * kStSlot + PR * kPwSlot + 2 * (SR + PR) * 8 + 16);
  Cursor& cp = *(&cs + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nitems = ntx * nty * nch;
  if (threadIdx.x == 0) {
    for (int s = 0; s < SR; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&st_full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&st_empty[s])), "r"(NW));
    }
    for (int s = 0; s < PR; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&pw_full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&pw_empty[s])), "r"(NW));
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    cs.it = cp.it = (int)blockIdx.x;
    if (cs.it < nitems) {
      const Item I = item_of(p, cs.it, ntx, nty, nch, kc);
      cs.kk = I.ka - 1;
      cp.kk = I.ka;
    }
    cs.n = cp.n = 0;
  }
  __syncthreads();

  // thread 0: issue stencil rows until `ts` positions and pointwise rows
  // until `tp` positions are issued (or the CTA's items end); a slot is
  // reused once every warp released its previous row.  False if a wait
  // gave up.
  auto produce = [&](long long ts, long long tp) -> bool {
    while (cs.n < ts && cs.it < nitems) {
      const int s = (int)(cs.n % SR);
      if (cs.n >= SR && !bar_wait(su32(&st_empty[s]), (uint32_t)(((cs.n / SR) - 1) & 1), abort_flag)) return false;
      const Item I = item_of(p, cs.it, ntx, nty, nch, kc);
      const uint32_t fb = su32(&st_full[s]);
      bar_expect(fb, kStTx);
      const uint32_t dst = su32(st_base + s * kStSlot);
#pragma unroll
      for (int f = 0; f < 6; ++f) tma3(dst + f * kStBox, &maps.st[f], I.i0 - 1, I.j0 - 1, cs.kk, fb);
      ++cs.n;
      if (++cs.kk > I.kb + 1) {
        cs.it += gridDim.x;
        if (cs.it < nitems) cs.kk = item_of(p, cs.it, ntx, nty, nch, kc).ka - 1;
      }
    }
    while (cp.n < tp && cp.it < nitems) {
      const int s = (int)(cp.n % PR);
      if (cp.n >= PR && !bar_wait(su32(&pw_empty[s]), (uint32_t)(((cp.n / PR) - 1) & 1), abort_flag)) return false;
      const Item I = item_of(p, cp.it, ntx, nty, nch, kc);
      const uint32_t fb = su32(&pw_full[s]);
      bar_expect(fb, kPwTx);
      const uint32_t dst = su32(pw_base + s * kPwSlot);
#pragma unroll
      for (int f = 0; f < 6; ++f) tma3(dst + f * kPgBox, &maps.pg[f], I.i0 - 1, I.j0, cp.kk, fb);
#pragma unroll
      for (int f = 0; f < 6; ++f) tma3(dst + 6 * kPgBox + f * kPiBox, &maps.pi[f], I.i0 - 1, I.j0 - 1, cp.kk - 1, fb);
      ++cp.n;
      if (++cp.kk > I.kb) {
        cp.it += gridDim.x;
        if (cp.it < nitems) cp.kk = item_of(p, cp.it, ntx, nty, nch, kc).ka;
      }
    }
    return true;
  };
  // on a failed wait: flag it; thread 0 lets the copies it issued land
  // before the CTA's shared memory is released
  auto give_up = [&]() {
    *abort_flag = 1;
    if (lane == 0) atomicExch(&dsc->wait_err, 1);
    if (threadIdx.x == 0) {
      for (long long n = std::max(0LL, cs.n - SR); n < cs.n; ++n)
        bar_wait(su32(&st_full[n % SR]), (uint32_t)((n / SR) & 1), nullptr);
      for (long long n = std::max(0LL, cp.n - PR); n < cp.n; ++n)
        bar_wait(su32(&pw_full[n % PR]), (uint32_t)((n / PR) & 1), nullptr);
    }
  };

  const int tx = lane, ty = warp;
  const double rho_avr = *rho_avr_p;
  long long ns = 0, np = 0;  // stream positions consumed
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = item_of(p, it, ntx, nty, nch, kc);
    const int i = I.i0 + tx, j = I.j0 + ty;
    const bool ok = i <= p.imax && j <= p.jmax;
    const long long sb = ns;   // stencil position of row ka-1
    const long long pb = np;   // pointwise position of row ka
    double dw_km1 = 0.;
    for (int k = I.ka; k <= I.kb; ++k) {
      const long long r = k - I.ka;
      // stencil through row k+2, pointwise through row k+1
      bool fail = false;
      if (threadIdx.x == 0) fail = !produce(sb + r + 4, pb + r + 2);
      __syncwarp();
      if (r == 0) {
        fail |= !bar_wait(su32(&st_full[sb % SR]), (uint32_t)((sb / SR) & 1), abort_flag);
        fail |= !bar_wait(su32(&st_full[(sb + 1) % SR]), (uint32_t)(((sb + 1) / SR) & 1), abort_flag);
      }
      const long long n2 = sb + r + 2;
      fail |= !bar_wait(su32(&st_full[n2 % SR]), (uint32_t)((n2 / SR) & 1), abort_flag);
      const long long pn = pb + r;
      fail |= !bar_wait(su32(&pw_full[pn % PR]), (uint32_t)((pn / PR) & 1), abort_flag);
      if (fail || *abort_flag) {
        give_up();
        return;
      }
      const double* sm_ = reinterpret_cast<const double*>(st_base + ((sb + r) % SR) * kStSlot);
      const double* s0_ = reinterpret_cast<const double*>(st_base + ((sb + r + 1) % SR) * kStSlot);
      const double* sp_ = reinterpret_cast<const double*>(st_base + (n2 % SR) * kStSlot);
      const unsigned char* pw = pw_base + (pn % PR) * kPwSlot;
      if (ok) {
        constexpr int FB = kStBox / 8;  // doubles per stencil box
        auto SL = [&](int dk) { return dk < 0 ? sm_ : (dk > 0 ? sp_ : s0_); };
        auto at = [&](int f, int di, int dj, int dk) {
          return SL(dk)[f * FB + (ty + 1 + dj) * SW + (tx + 1 + di)];
        };
        auto U = [&](int di, int dj, int dk) { return at(0, di, dj, dk); };
        auto V = [&](int di, int dj, int dk) { return at(1, di, dj, dk); };
        auto W = [&](int di, int dj, int dk) { return at(2, di, dj, dk); };
        auto M = [&](int di, int dj, int dk) { return at(3, di, dj, dk); };
        auto PH = [&](int di, int dj, int dk) { return 2. * at(4, di, dj, dk) - at(5, di, dj, dk); };
        const double* pg = reinterpret_cast<const double*>(pw);
        const double* pi = reinterpret_cast<const double*>(pw + 6 * kPgBox);
        const int og = ty * SW + tx + 1, oi = ty * TX + tx;
        constexpr int GB = kPgBox / 8, IB = kPiBox / 8;
        const double qx = pg[og], qy = pg[GB + og], qz = pg[2 * GB + og];
        const double qxo = pg[3 * GB + og], qyo = pg[4 * GB + og], qzo = pg[5 * GB + og];
        const double ru = pi[oi], rv = pi[IB + oi], rw = pi[2 * IB + oi];
        const double ou = pi[3 * IB + oi], ov = pi[4 * IB + oi], ow = pi[5 * IB + oi];
        const double ph0 = PH(0, 0, 0);
        const double Ru = rhs_u<double>(p, U, V, W, M, ru, rho_avr);
        const double Rv = rhs_v<double>(p, U, V, W, M, rv, rho_avr);
        const double Rw = rhs_w<double>(p, U, V, W, M, rw, rho_avr);
        const double du = ab2_update_v(p, U(0, 0, 0), Ru, ou, ru, PH(1, 0, 0), ph0, 2. * qx - qxo, p.dxi);
        double dv = ab2_update_v(p, V(0, 0, 0), Rv, ov, rv, PH(0, 1, 0), ph0, 2. * qy - qyo, p.dyi);
        if (p.forceytot != 0.) dv = dv - (p.forceytot * p.dt) / rv;
        double dw = ab2_update_v(p, W(0, 0, 0), Rw, ow, rw, PH(0, 0, 1), ph0, 2. * qz - qzo, p.dzi);
        const long long q = idxI(p, i, j, k);
        duold_out[q] = Ru;
        dvold_out[q] = Rv;
        dwold_out[q] = Rw;
        if (k == p.kmax - 1) dw_km1 = dw;
        if (k == p.kmax) dw = 0.;
        putC(p, dudt, i, j, k, du);
        putC(p, dvdt, i, j, k, dv);
        putC(p, dwdt, i, j, k, dw);
        if (k == 1) {
          putC(p, dudt, i, j, 0, -du);
          putC(p, dvdt, i, j, 0, 2. * p.v_lower - dv);
          putC(p, dwdt, i, j, 0, 0.);
        }
        if (k == p.kmax) {
          putC(p, dudt, i, j, p.k1, -du);
          putC(p, dvdt, i, j, p.k1, 2. * p.v_upper - dv);
          putC(p, dwdt, i, j, p.k1, dw_km1);
        }
      }
      // this warp is done with stencil row k-1 and pointwise row k
      __syncwarp();
      if (lane == 0) {
        bar_arrive(su32(&st_empty[(sb + r) % SR]));
        bar_arrive(su32(&pw_empty[pn % PR]));
      }
    }
    const long long nr = I.kb - I.ka + 1;
    __syncwarp();
    if (lane == 0) {  // rows kb and kb+1 are not needed by the next item
      bar_arrive(su32(&st_empty[(sb + nr) % SR]));
      bar_arrive(su32(&st_empty[(sb + nr + 1) % SR]));
    }
    ns = sb + nr + 2;
    np = pb + nr;
  }
}

// ------------------------------------------------------------ tensor maps
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

bool encode3(CUtensorMap* m, const double* base, int nx, int ny, int nz, int bx, int by) {
  auto fn = encode_fn();
  if (!fn) return false;
  if (reinterpret_cast<uintptr_t>(base) % 16) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * 8, (cuuint64_t)nx * ny * 8};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  if (strides[0] % 16 || strides[1] % 16) return false;
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the 18 input pointers in the maps' order
void map_keys(const MomArgs& a, const void* k[18]) {
  const double* all[18] = {a.u,  a.v,  a.w,  a.miu,   a.pnew,  a.pold,  a.px,    a.py,    a.pz,
                           a.pxold, a.pyold, a.pzold, a.rho_u, a.rho_v, a.rho_w, a.duold, a.dvold, a.dwold};
  for (int q = 0; q < 18; ++q) k[q] = all[q];
}

bool build_maps(Ctx& c, const MomArgs& a, Ab2Maps* m) {
  const Params& P = c.P;
  const double* st[6] = {a.u, a.v, a.w, a.miu, a.pnew, a.pold};
  const double* pg[6] = {a.px, a.py, a.pz, a.pxold, a.pyold, a.pzold};
  const double* pi[6] = {a.rho_u, a.rho_v, a.rho_w, a.duold, a.dvold, a.dwold};
  for (int f = 0; f < 6; ++f) {
    if (!encode3(&m->st[f], st[f], P.nCx, P.nCy, P.nCz, SW, SH)) return false;
    if (!encode3(&m->pg[f], pg[f], P.nCx, P.nCy, P.nCz, SW, TY)) return false;
    if (!encode3(&m->pi[f], pi[f], P.imax, P.jmax, P.kmax, TX, TY)) return false;
  }
  return true;
}

}  // namespace

// The TMA predictor when it applies (FP64 fields, imax even so every row
// pitch is a multiple of 16 bytes, tensor maps encodable); false leaves the
// launch to the caller's k_ab2.
bool ab2_tma_launch(Ctx& c, const MomArgs& a, int o) {
  if (c.P.f32 || c.ab2_ring || c.ab2_tma_failed || (c.P.imax & 1) || c.P.kmax < 2) return false;
  static_assert(sizeof(Ab2Maps) <= sizeof(c.ab2_maps[0]), "tensor-map cache too small");
  const void* key[18];
  map_keys(a, key);
  int slot = -1;
  for (int q = 0; q < c.ab2_nmaps && slot < 0; ++q)
    if (std::memcmp(c.ab2_keys[q], key, sizeof(key)) == 0) slot = q;
  if (slot < 0) {  // encode into a free slot, else the oldest one
    slot = c.ab2_nmaps < 4 ? c.ab2_nmaps++ : c.ab2_next;
    c.ab2_next = (slot + 1) % 4;
    std::memset(c.ab2_keys[slot], 0, sizeof(key));
    if (!build_maps(c, a, reinterpret_cast<Ab2Maps*>(c.ab2_maps[slot]))) {
      c.ab2_tma_failed = true;
      return false;
    }
    std::memcpy(c.ab2_keys[slot], key, sizeof(key));
  }
  Ab2Maps* maps = reinterpret_cast<Ab2Maps*>(c.ab2_maps[slot]);
  static unsigned attr = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr & (1u << (dev & 31)))) {
    if (cudaFuncSetAttribute(k_ab2_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTma) != cudaSuccess)
      return false;
    attr |= 1u << (dev & 31);
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int ntx = (c.P.imax + TX - 1) / TX, nty = (c.P.jmax + TY - 1) / TY;
  const int kc = std::min(kRowsPerItem, c.P.kmax);
  const int nch = std::max(1, c.P.kmax / kc);
  const int nitems = ntx * nty * nch;
  const int grid = std::min(nsm, nitems);
  k_ab2_tma<<<grid, kThreadsTma, kSmemTma, c.s>>>(*maps, c.P, a.rho_avr, c.dudt, c.dvdt, c.dwdt, c.duold[o],
                                                   c.dvold[o], c.dwold[o], c.dsc, ntx, nty, nch,
                                                   nch == 1 ? c.P.kmax : kc);
  return true;
}

}  // namespace icls
