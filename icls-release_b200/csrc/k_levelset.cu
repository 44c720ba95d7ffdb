// k_levelset.cu — level-set kernels of the ICLS hot path (FP64, -fmad=false).
//
//   tube_construction  levelset.f90:87-197
//   HOUC5_nb/WENO5_nb  hyperPDE.f90:397-800, fused with RK_nb
//                      levelset.f90:342-367 and boundsls bound.f90:386-483
//   ls_reinit          levelset.f90:619-882 with WENO5_reinit/WENO5_deri
//                      hyperPDE.f90:2646-2746, 2932-3197
//   inflation          levelset.f90:407-582
//   update_materials   misc.f90:79-290 with Heaviside 'trig' misc.f90:297-464
//
// Halo handling: instead of a separate boundsls pass, a thread computes an
// interior column and writes it together with its periodic halo images;
// the wall rows k=0 and k=k1 are the linear extrapolation of the two
// interior values next to them, evaluated by the thread that computes
// those.  This reproduces boundsls (z-extrapolation, then periodic x, then
// periodic y) exactly, because the inputs satisfy the periodic halo
// invariant.
//
// Sweep regions: after tube_construction clips the level set to +-6dz,
// every cell outside a drop's band holds the same far-field value, and
// every kernel maps a uniform neighbourhood to a uniform value (the
// stencils of a constant field are exactly zero).  Each per-drop kernel
// therefore sweeps only a region around the band (periodic column spans in
// x and y, rows in z) and writes the far-field value, replayed on the host
// with the same arithmetic, into a 3-cell apron around it; reads never
// leave the region plus apron.  All drops of a step go through one launch
// per stage (batch.cuh).
//
// In-place stages: the last RK stage may write the array it takes as its
// pointwise base (phi0): a thread reads phi0 only in its own column, and
// it writes a wall row only after it has computed the rows it extrapolates.
#include <algorithm>
#include <climits>

#include "batch.cuh"

namespace icls {

namespace {

constexpr int NT = TBX * TBY;
const dim3 kTile(TBX, TBY, 1);
const dim3 kBlock(BX, BY, 1);

// T is the type the level-set fields are stored and computed in: double
// for the reference form, float for the precision form.  TC(x) is the
// constant x in T.
#define TC(x) static_cast<T>(x)

template <typename T>
__device__ __forceinline__ T clipNB(T x, T NB) {
  return x > NB ? NB : (x < -NB ? -NB : x);
}
__device__ __forceinline__ bool interior(const Params& p, int i, int j, int k) {
  return i >= 1 && i <= p.imax && j >= 1 && j <= p.jmax && k >= 1 && k <= p.kmax;
}

// ---------------------------------------------------------------- band extents
// The band box a tube_construction sweep of the whole array would measure
// (the cells of rows -2..k1+2 whose clipped value differs from +NB, rows 0
// and k1 by the wall extrapolation), in the same two frames per periodic
// axis, without writing anything: one thread per (i,j) column.
template <typename T>
__global__ void __launch_bounds__(NT) k_band_extents(Params p, const T* __restrict__ phi, int l,
                                                     int* __restrict__ bbox_lo, int* __restrict__ bbox_hi) {
  const long long q = blockIdx.x * (long long)NT + threadIdx.x;
  int lo[5] = {INT_MAX, INT_MAX, INT_MAX, INT_MAX, INT_MAX};
  int hi[5] = {INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN};
  if (q < (long long)p.imax * p.jmax) {
    const int i = (int)(q % p.imax) + 1, j = (int)(q / p.imax) + 1;
    const int hx = p.imax / 2, hy = p.jmax / 2;
    const int ib = i + hx > p.imax ? i + hx - p.imax : i + hx;
    const int jb = j + hy > p.jmax ? j + hy - p.jmax : j + hy;
    const T NB = TC(p.NB);
    const long long sz = (long long)p.nLx * p.nLy, c0 = idxL(p, i, j, 0);
    for (int k = -2; k <= p.k1 + 2; ++k) {
      T val;
      if (k == 0)
        val = TC(2.) * clipNB(phi[c0 + sz], NB) - clipNB(phi[c0 + 2 * sz], NB);
      else if (k == p.k1)
        val = TC(2.) * clipNB(phi[c0 + p.kmax * sz], NB) - clipNB(phi[c0 + (p.kmax - 1) * sz], NB);
      else
        val = clipNB(phi[c0 + k * sz], NB);
      if (val != NB) {
        lo[0] = min(lo[0], i); hi[0] = max(hi[0], i);
        lo[1] = min(lo[1], ib); hi[1] = max(hi[1], ib);
        lo[2] = min(lo[2], j); hi[2] = max(hi[2], j);
        lo[3] = min(lo[3], jb); hi[3] = max(hi[3], jb);
        lo[4] = min(lo[4], k); hi[4] = max(hi[4], k);
      }
    }
  }
  for (int a = 0; a < 5; ++a) {
    int lv = lo[a], h = hi[a];
    for (int o = 16; o > 0; o >>= 1) {
      lv = min(lv, __shfl_down_sync(0xffffffffu, lv, o));
      h = max(h, __shfl_down_sync(0xffffffffu, h, o));
    }
    if ((threadIdx.x & 31) == 0 && lv != INT_MAX) {
      atomicMin(&bbox_lo[5 * l + a], lv);
      atomicMax(&bbox_hi[5 * l + a], h);
    }
  }
}

// ---------------------------------------------------------------- tube
// Clip to +-NB (levelset.f90:120-128) and the band mask (130-160) over the
// tasks' regions.  phi0 holds valid data on vin's written cells, bgin
// (rows 0..k1) or bggin (ghost rows) elsewhere.  Counts the band per drop
// and records the extent of the cells whose clipped value is not +NB:
// bbox_lo[5 l + a], bbox_hi[5 l + a] for a = x, x shifted by imax/2, y, y
// shifted by jmax/2, z.  A far-field cell is outside the band only if all
// 15 axial neighbours clip to +-NB, so the test stops at the first that
// does not (the reference's sums of |clip|-NB <= 0 are zero exactly then).
template <typename T>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 5 : 4)) k_tube(Params p, const __grid_constant__ LsBatch B,
                                             long long* __restrict__ cnt, int* __restrict__ bbox_lo,
                                             int* __restrict__ bbox_hi) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const T NB = TC(p.NB);
  const T* __restrict__ in = cT<T>(t.phi0);
  T* __restrict__ out = mT<T>(t.out);
  const T bgin = TC(t.bgin), bggin = TC(t.bggin);
  int band = 0;
  int lo[5] = {INT_MAX, INT_MAX, INT_MAX, INT_MAX, INT_MAX};
  int hi[5] = {INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN};
  // The band test reads, per row, in-band flags |clip(phi)| != NB of the
  // tile's columns and a 2-column halo from a shared-memory plane (double
  // buffered, one barrier per row) and of its own column's rows k-2..k+2
  // from a register window.  Every flag comes from the input as the
  // original reads did: the input region's value where it holds the
  // column (tested on the wrapped column index) and row, else its far-field
  // value.
  __shared__ uint8_t F[2][TBY + 4][TBX + 4];
  const int tx = (int)threadIdx.x, ty = (int)threadIdx.y, tid = tx + TBX * ty;
  const int X0 = c.X - tx, Y0 = c.Y - ty;  // the tile's first column in region coordinates
  auto wrapn = [](int v, int n) { v %= n; return v < 0 ? v + n : v; };
  auto column = [&](int X, int Y, int& iw, int& jw, bool& held) {
    iw = wrapn(t.r.xa - 1 + X, p.imax) + 1;
    jw = wrapn(t.r.ya - 1 + Y, p.jmax) + 1;
    held = span_has(t.vin.xa, t.vin.xn, p.imax, iw) && span_has(t.vin.ya, t.vin.yn, p.jmax, jw);
  };
  auto rdo = [&](long long at, bool held, int k) -> T {
    return (held && k >= t.vin.z0 && k <= t.vin.z1) ? in[at] : ((k < 0 || k > p.k1) ? bggin : bgin);
  };
  auto flag = [&](T v) -> uint8_t { return fabs(clipNB(v, NB)) != NB ? 1 : 0; };
  const long long sz = (long long)p.nLx * p.nLy;
  // this thread's column (in or out of the region) and its halo cell, if any
  int iw, jw, hi_w = 0, hj_w = 0, hxs = 0, hys = 0;
  bool held, hheld = false;
  column(c.X, c.Y, iw, jw, held);
  const bool has_halo = tid < 4 * TBY + 4 * TBX;  // 4 halo columns x TBY rows, 4 halo rows x TBX columns
  if (has_halo) {
    int xo, yo;
    if (tid < 4 * TBY) {
      const int side = tid / TBY;  // columns -2, -1, TBX, TBX+1
      xo = side < 2 ? side - 2 : TBX + side - 2;
      yo = tid % TBY;
    } else {
      const int u = tid - 4 * TBY, side = u / TBX;  // rows -2, -1, TBY, TBY+1
      xo = u % TBX;
      yo = side < 2 ? side - 2 : TBY + side - 2;
    }
    column(X0 + xo, Y0 + yo, hi_w, hj_w, hheld);
    hxs = xo + 2;
    hys = yo + 2;
  }
  const long long cw = idxL(p, iw, jw, 0), hw = idxL(p, hi_w, hj_w, 0);
  // z window: flags of this column at rows k-2 .. k+2 (slots 1..4 hold rows
  // ka-2..ka+1; each row shifts down one slot and reads row k+2 into slot 4)
  uint8_t fz[5];
  fz[0] = 0;
#pragma unroll
  for (int d = -2; d <= 1; ++d) fz[d + 3] = flag(rdo(cw + (c.ka + d) * sz, held, c.ka + d));
  // the values a row turns into flags (row k+2 of this column, row k of the
  // halo cell) were read one row earlier, so a barrier waits on no fresh load
  T nz = rdo(cw + (c.ka + 2) * sz, held, c.ka + 2);
  T nh = has_halo ? rdo(hw + c.ka * sz, hheld, c.ka) : bgin;
  const int i = c.i, j = c.j;
  const int hx = p.imax / 2, hy = p.jmax / 2;
  const int ib = i + hx > p.imax ? i + hx - p.imax : i + hx;
  const int jb = j + hy > p.jmax ? j + hy - p.jmax : j + hy;
  const bool colin = held;
  for (int k = c.ka; k <= c.kb; ++k) {
#pragma unroll
    for (int d = 0; d < 4; ++d) fz[d] = fz[d + 1];
    fz[4] = flag(nz);
    nz = rdo(cw + (k + 3) * sz, held, k + 3);
    const int buf = k & 1;
    F[buf][ty + 2][tx + 2] = fz[2];
    if (has_halo) {
      F[buf][hys][hxs] = flag(nh);
      nh = rdo(hw + (k + 1) * sz, hheld, k + 1);
    }
    __syncthreads();
    if (c.ok) {
      T val;
      const long long c0 = idxL(p, i, j, k);
      if (!computed(c, t.r, k)) {
        val = clipNB((k < 0 || k > p.k1) ? bggin : bgin, NB);
      } else {
        if (k == 0)
          val = TC(2.) * clipNB(rdo(c0 + sz, colin, 1), NB) - clipNB(rdo(c0 + 2 * sz, colin, 2), NB);
        else if (k == p.k1)
          val = TC(2.) * clipNB(rdo(c0 - sz, colin, p.kmax), NB) - clipNB(rdo(c0 - 2 * sz, colin, p.kmax - 1), NB);
        else
          val = clipNB(rdo(c0, colin, k), NB);
        if (k >= 1 && k <= p.kmax) {
          const uint8_t(&Fp)[TBY + 4][TBX + 4] = F[buf];
          const int m = (fz[2] | Fp[ty + 2][tx] | Fp[ty + 2][tx + 1] | Fp[ty + 2][tx + 3] | Fp[ty + 2][tx + 4] |
                         Fp[ty][tx + 2] | Fp[ty + 1][tx + 2] | Fp[ty + 3][tx + 2] | Fp[ty + 4][tx + 2] | fz[0] |
                         fz[1] | fz[3] | fz[4]) != 0;
          t.mask[idxI(p, i, j, k)] = (uint8_t)m;
          band += m;
        }
        if (val != NB) {
          lo[0] = min(lo[0], i); hi[0] = max(hi[0], i);
          lo[1] = min(lo[1], ib); hi[1] = max(hi[1], ib);
          lo[2] = min(lo[2], j); hi[2] = max(hi[2], j);
          lo[3] = min(lo[3], jb); hi[3] = max(hi[3], jb);
          lo[4] = min(lo[4], k); hi[4] = max(hi[4], k);
        }
      }
      putL(p, out, i, j, k, val);
    }
  }
  const int bs = block_sum<int, NT>(band);
  if (flat_tid() == 0 && bs) atomicAdd((unsigned long long*)(cnt + t.l), (unsigned long long)bs);
  for (int a = 0; a < 5; ++a) {
    int l = lo[a], h = hi[a];
    for (int o = 16; o > 0; o >>= 1) {
      l = min(l, __shfl_down_sync(0xffffffffu, l, o));
      h = max(h, __shfl_down_sync(0xffffffffu, h, o));
    }
    if ((flat_tid() & 31) == 0 && l != INT_MAX) {
      atomicMin(&bbox_lo[5 * t.l + a], l);
      atomicMax(&bbox_hi[5 * t.l + a], h);
    }
  }
}

// ------------------------------------------------------- advection RHS
// The 19 values of the axial stencil of a cell (the centre and offsets
// -3..3 along each axis).
template <typename T>
struct Axial19 {
  T c, x[7], y[7], z[7];  // x[d + 3] = phi at offset d along x (x[3] == c), likewise y, z
};

// dfdt of HOUC5_nb (hyperPDE.f90:397-495) or WENO5_nb (503-800) at row k
// from its axial stencil S
template <int SCHEME, int PW = -1, typename T>
__device__ __forceinline__ T adv_rhs(const Params& p, const Axial19<T>& S, T vu, T vv, T vw, int k) {
#define PX(d) S.x[(d) + 3]
#define PY(d) S.y[(d) + 3]
#define PZ(d) S.z[(d) + 3]
  T udfdx, vdfdy, wdfdz, dfx, dfy, dfz;
  if (SCHEME == ICLS_HOUC5) {
    if (p.TwoD) {
      udfdx = TC(0.);
    } else {
      if (vu >= TC(0.))
        dfx = houc5_pos(PX(-3), PX(-2), PX(-1), PX(0), PX(1), PX(2));
      else
        dfx = houc5_neg(PX(3), PX(2), PX(1), PX(0), PX(-1), PX(-2));
      udfdx = -divx<PW>(p, vu * dfx);
    }
    if (vv >= TC(0.))
      dfy = houc5_pos(PY(-3), PY(-2), PY(-1), PY(0), PY(1), PY(2));
    else
      dfy = houc5_neg(PY(3), PY(2), PY(1), PY(0), PY(-1), PY(-2));
    vdfdy = -divy<PW>(p, vv * dfy);
  } else {
    if (p.TwoD) {
      udfdx = TC(0.);
    } else {
      if (vu >= TC(0.))
        dfx = weno5(divx<PW>(p, PX(-2) - PX(-3)), divx<PW>(p, PX(-1) - PX(-2)), divx<PW>(p, PX(0) - PX(-1)),
                    divx<PW>(p, PX(1) - PX(0)), divx<PW>(p, PX(2) - PX(1)));
      else
        dfx = weno5(divx<PW>(p, PX(3) - PX(2)), divx<PW>(p, PX(2) - PX(1)), divx<PW>(p, PX(1) - PX(0)),
                    divx<PW>(p, PX(0) - PX(-1)), divx<PW>(p, PX(-1) - PX(-2)));
      udfdx = -(vu * dfx);
    }
    // y uses dx, as in the reference (hyperPDE.f90:622-626)
    if (vv >= TC(0.))
      dfy = weno5(divx<PW>(p, PY(-2) - PY(-3)), divx<PW>(p, PY(-1) - PY(-2)), divx<PW>(p, PY(0) - PY(-1)),
                  divx<PW>(p, PY(1) - PY(0)), divx<PW>(p, PY(2) - PY(1)));
    else
      dfy = weno5(divx<PW>(p, PY(3) - PY(2)), divx<PW>(p, PY(2) - PY(1)), divx<PW>(p, PY(1) - PY(0)),
                  divx<PW>(p, PY(0) - PY(-1)), divx<PW>(p, PY(-1) - PY(-2)));
    vdfdy = -(vv * dfy);
  }
  if (k > 2 && k < p.kmax - 1) {
    if (SCHEME == ICLS_HOUC5) {
      if (vw >= TC(0.))
        dfz = houc5_pos(PZ(-3), PZ(-2), PZ(-1), PZ(0), PZ(1), PZ(2));
      else
        dfz = houc5_neg(PZ(3), PZ(2), PZ(1), PZ(0), PZ(-1), PZ(-2));
      wdfdz = -divz<PW>(p, vw * dfz);
    } else {
      if (vw >= TC(0.))
        dfz = weno5(divz<PW>(p, PZ(-2) - PZ(-3)), divz<PW>(p, PZ(-1) - PZ(-2)), divz<PW>(p, PZ(0) - PZ(-1)),
                    divz<PW>(p, PZ(1) - PZ(0)), divz<PW>(p, PZ(2) - PZ(1)));
      else
        dfz = weno5(divz<PW>(p, PZ(3) - PZ(2)), divz<PW>(p, PZ(2) - PZ(1)), divz<PW>(p, PZ(1) - PZ(0)),
                    divz<PW>(p, PZ(0) - PZ(-1)), divz<PW>(p, PZ(-1) - PZ(-2)));
      wdfdz = -(vw * dfz);
    }
  } else if (k == 2 || k == p.kmax - 1) {  // HOUC3 near the walls
    if (vw >= TC(0.))
      dfz = ((TC(1. / 6.) * PZ(-2) - PZ(-1)) + TC(1. / 2.) * PZ(0)) + TC(1. / 3.) * PZ(1);
    else
      dfz = ((-(TC(1. / 6.) * PZ(2)) + PZ(1)) - TC(1. / 2.) * PZ(0)) - TC(1. / 3.) * PZ(-1);
    wdfdz = -divz<PW>(p, vw * dfz);
  } else {  // first-order upwinding at k=1,kmax
    if (vw >= TC(0.)) dfz = PZ(0) - PZ(-1);
    else dfz = PZ(1) - PZ(0);
    wdfdz = -divz<PW>(p, vw * dfz);
  }
#undef PX
#undef PY
#undef PZ
  return (udfdx + vdfdy) + wdfdz;
}
template <int SCHEME, typename T, int PW>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 5 : 4)) k_adv_stage(Params p, const __grid_constant__ LsBatch B, int stage1,
                                                     double a_, double bb_, double fdt_, const T* __restrict__ vu,
                                                     const T* __restrict__ vv, const T* __restrict__ vw) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok) return;
  const T a = TC(a_), bb = TC(bb_), fdt = TC(fdt_);
  const int i = c.i, j = c.j;
  // This column's storage, and that of its periodic images in out, from
  // row 0; row k is `k * sz` further (32-bit offsets within one array).
  const int sy = p.nLx, sz = p.nLx * p.nLy, szI = p.imax * p.jmax;
  const long long col = idxL(p, i, j, 0);
  const T* f0c = cT<T>(t.phi0) + col;
  const T* fsc = cT<T>(t.phis) + col;
  T* out = mT<T>(t.out);
  T* const o0 = out + col;
  const int ii = image_of<3>(i, p.imax), jj = image_of<3>(j, p.jmax);
  T* const o1 = ii != INT_MIN ? out + idxL(p, ii, j, 0) : nullptr;
  T* const o2 = jj != INT_MIN ? out + idxL(p, i, jj, 0) : nullptr;
  T* const o3 = (ii != INT_MIN && jj != INT_MIN) ? out + idxL(p, ii, jj, 0) : nullptr;
  const long long qc = idxI(p, i, j, 1);  // row k at qc + (k - 1) * szI
  auto put = [&](int k, T v) {
    const int o = k * sz;
    o0[o] = v;
    if (o1) o1[o] = v;
    if (o2) o2[o] = v;
    if (o3) o3[o] = v;
  };
  T v1 = TC(0.), v2 = TC(0.), vkm = TC(0.), vk = TC(0.);
  bool wall0 = false;
  for (int k = c.ka; k <= c.kb; ++k) {
    if (!computed(c, t.r, k)) {
      put(k, (k < 0 || k > p.k1) ? TC(t.bgg) : TC(t.bg));
      continue;
    }
    if (k == 0) {  // written once rows 1 and 2 are known
      wall0 = true;
      continue;
    }
    T val;
    if (k == p.k1) {
      val = TC(2.) * vk - vkm;
    } else {
      // every operand (phi0, phis' axial stencil, the band flag and the
      // velocities) is read first, so one memory latency is exposed per row;
      // the stencil result is used on band cells only
      const int o = k * sz;
      const T f0 = f0c[o];
      if (!(k >= 1 && k <= p.kmax)) {
        val = stage1 ? f0 : a * f0 + bb * fsc[o];
      } else {
        const long long q = qc + (long long)(k - 1) * szI;
        const uint8_t m = t.mask[q];
        const T u = vu[q], v = vv[q], w = vw[q];
        const T* f = fsc + o;
        Axial19<T> S;
        S.c = f[0];
#pragma unroll
        for (int d = -3; d <= 3; ++d) {
          if (d == 0) continue;
          S.x[d + 3] = f[d];
          S.y[d + 3] = f[d * sy];
          S.z[d + 3] = f[d * sz];
        }
        S.x[3] = S.y[3] = S.z[3] = S.c;
        val = stage1 ? f0 : a * f0 + bb * S.c;
        if (m) val = val + fdt * adv_rhs<SCHEME, PW>(p, S, u, v, w, k);
      }
      if (k == 1) v1 = val;
      if (k == 2) v2 = val;
      if (k == p.kmax - 1) vkm = val;
      if (k == p.kmax) vk = val;
    }
    put(k, val);
    if (k == 2 && wall0) put(0, TC(2.) * v1 - v2);
  }
}

// ------------------------------------------------- band-list advection
// One RK stage of k_adv_stage split in three launches over the same tasks,
// with the same arithmetic per cell (bit-identical):
//   k_adv_base   every written cell its value without the transport term:
//                the far field outside the computed part, else f0 (stage
//                1) or a f0 + bb fs; the wall rows 0 and k1 are left
//   k_adv_band   adds fdt * dfdt on the band cells of a compacted list
//                (k_band_list, built once after tube_construction for all
//                three stages): full warps, and no lane walks a clipped
//                column only to copy it
//   k_adv_walls  rows 0 and k1 from the finished rows next to them, under
//                the conditions k_adv_stage writes them
// The list holds the computed interior cells whose band flag is set, as
// (i-1) | (j-1) << 12 | task << 24 and k.
struct BandCell {
  unsigned ijt;
  int k;
};

template <typename T>
__global__ void __launch_bounds__(NT) k_band_list(Params p, const __grid_constant__ LsBatch B,
                                                  BandCell* __restrict__ list, int* __restrict__ count, int cap) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const unsigned lane = threadIdx.x & 31u;
  const long long q0 = c.ok ? idxI(p, c.i, c.j, 1) : 0;
  const long long szI = (long long)p.imax * p.jmax;
  // every lane of a block walks the same rows, so the ballots line up
  for (int k = max(c.ka, 1); k <= min(c.kb, p.kmax); ++k) {
    const bool take = c.ok && computed(c, t.r, k) && t.mask[q0 + (k - 1) * szI];
    const unsigned msk = __ballot_sync(0xffffffffu, take);
    if (!msk) continue;
    int base = 0;
    if (lane == (unsigned)(__ffs(msk) - 1)) base = atomicAdd(count, __popc(msk));
    base = __shfl_sync(0xffffffffu, base, __ffs(msk) - 1);
    const int slot = base + __popc(msk & ((1u << lane) - 1u));
    if (take && slot < cap)
      list[slot] = BandCell{(unsigned)(c.i - 1) | ((unsigned)(c.j - 1) << 12) | ((unsigned)ti << 24), k};
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k_adv_base(Params p, const __grid_constant__ LsBatch B, int stage1, double a_,
                                                 double bb_) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok) return;
  const T a = TC(a_), bb = TC(bb_);
  const T* __restrict__ f0c = cT<T>(t.phi0);
  const T* __restrict__ fsc = cT<T>(t.phis);
  T* out = mT<T>(t.out);
  for (int k = c.ka; k <= c.kb; ++k) {
    if (!computed(c, t.r, k)) {
      putL(p, out, c.i, c.j, k, (k < 0 || k > p.k1) ? TC(t.bgg) : TC(t.bg));
      continue;
    }
    if (k == 0 || k == p.k1) continue;  // k_adv_walls
    const long long o = idxL(p, c.i, c.j, k);
    const T f0 = f0c[o];
    putL(p, out, c.i, c.j, k, stage1 ? f0 : a * f0 + bb * fsc[o]);
  }
}

template <int SCHEME, typename T, int PW>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 4 : 3))
    k_adv_band(Params p, const __grid_constant__ LsBatch B, const BandCell* __restrict__ list,
               const int* __restrict__ count, double fdt_, const T* __restrict__ vu, const T* __restrict__ vv,
               const T* __restrict__ vw) {
  const int n = (int)(blockIdx.x * NT + threadIdx.x);
  if (n >= *count) return;
  const BandCell bc = list[n];
  const int i = (int)(bc.ijt & 0xFFFu) + 1, j = (int)((bc.ijt >> 12) & 0xFFFu) + 1, ti = (int)(bc.ijt >> 24);
  const int k = bc.k;
  const LsTask& t = B.t[ti];
  const T fdt = TC(fdt_);
  const long long sy = p.nLx, sz = (long long)p.nLx * p.nLy;
  const long long o = idxL(p, i, j, k);
  const long long q = idxI(p, i, j, k);
  const T* __restrict__ f = cT<T>(t.phis) + o;
  T* out = mT<T>(t.out);
  const T base = out[o];  // k_adv_base's value of this cell
  Axial19<T> S;
  S.c = f[0];
#pragma unroll
  for (int d = -3; d <= 3; ++d) {
    if (d == 0) continue;
    S.x[d + 3] = f[d];
    S.y[d + 3] = f[d * sy];
    S.z[d + 3] = f[d * sz];
  }
  S.x[3] = S.y[3] = S.z[3] = S.c;
  putL(p, out, i, j, k, base + fdt * adv_rhs<SCHEME, PW>(p, S, vu[q], vv[q], vw[q], k));
}

template <typename T>
__global__ void __launch_bounds__(NT) k_adv_walls(Params p, const __grid_constant__ LsBatch B) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok) return;
  T* out = mT<T>(t.out);
  auto at = [&](int k) { return out[idxL(p, c.i, c.j, k)]; };
  // the rows of this block's chunk that were computed, as k_adv_stage sees them
  auto row = [&](int k) { return k >= c.ka && k <= c.kb && computed(c, t.r, k); };
  // k = 0: written when row 2 of the same chunk was computed, from rows 1
  // (0 if not computed) and 2
  if (row(0) && row(2)) putL(p, out, c.i, c.j, 0, TC(2.) * (row(1) ? at(1) : TC(0.)) - at(2));
  // k = k1: from rows kmax and kmax-1 of the same chunk (0 where not computed)
  if (row(p.k1)) {
    const T vk = row(p.kmax) ? at(p.kmax) : TC(0.);
    const T vkm = row(p.kmax - 1) ? at(p.kmax - 1) : TC(0.);
    putL(p, out, c.i, c.j, p.k1, TC(2.) * vk - vkm);
  }
}

// ------------------------------------------------------------ reinit
// sgn(phi_0) of ls_reinit (levelset.f90:668-678)
template <typename T>
__device__ __forceinline__ T reinit_sgn(const Params& p, T p0) {
  const T dz = TC(p.dz);
  if (p0 < -dz) return TC(-1.);
  if (p0 > dz) return TC(1.);
  return p0 / sqrt(p0 * p0 + dz * dz);
}

// RHS of WENO5_reinit at an interior cell (hyperPDE.f90:2646-2746)
template <int PW, typename T>
__device__ __forceinline__ T reinit_rhs(const Params& p, const T* __restrict__ phi, const T* __restrict__ orig,
                                        int i, int j, int k) {
  const long long c = idxL(p, i, j, k);
  if (!(fabs(phi[c]) < TC(p.NB + p.dz))) return TC(0.);
  const long long sx = 1, sy = p.nLx, sz = (long long)p.nLx * p.nLy;
#define PH(o) phi[c + (o)]
  // A uniform neighbourhood (most of a drop's region is clipped far field):
  // every difference below is exactly +0, so every WENO5 derivative, the
  // Godunov choices and the gradient norm are exactly 0 and the right-hand
  // side is sgn * (1 - sqrt(0)) = sgn, bit for bit.  The test reads the
  // three axial neighbours each way (a superset of what the wall rows use).
  {
    const T c0 = PH(0);
    bool uni = true;
#pragma unroll
    for (int d = 1; d <= 3; ++d)
      uni = uni & (PH(d * sx) == c0) & (PH(-d * sx) == c0) & (PH(d * sy) == c0) & (PH(-d * sy) == c0) &
            (PH(d * sz) == c0) & (PH(-d * sz) == c0);
    if (uni) return reinit_sgn(p, orig[c]);
  }
  T A = TC(0.), B = TC(0.), C, D, E, F;
  if (!p.TwoD) {
    A = weno5(divx<PW>(p, PH(-2 * sx) - PH(-3 * sx)), divx<PW>(p, PH(-sx) - PH(-2 * sx)), divx<PW>(p, PH(0) - PH(-sx)),
              divx<PW>(p, PH(sx) - PH(0)), divx<PW>(p, PH(2 * sx) - PH(sx)));
    B = weno5(divx<PW>(p, PH(3 * sx) - PH(2 * sx)), divx<PW>(p, PH(2 * sx) - PH(sx)), divx<PW>(p, PH(sx) - PH(0)),
              divx<PW>(p, PH(0) - PH(-sx)), divx<PW>(p, PH(-sx) - PH(-2 * sx)));
  }
  C = weno5(divx<PW>(p, PH(-2 * sy) - PH(-3 * sy)), divx<PW>(p, PH(-sy) - PH(-2 * sy)), divx<PW>(p, PH(0) - PH(-sy)),
            divx<PW>(p, PH(sy) - PH(0)), divx<PW>(p, PH(2 * sy) - PH(sy)));
  D = weno5(divx<PW>(p, PH(3 * sy) - PH(2 * sy)), divx<PW>(p, PH(2 * sy) - PH(sy)), divx<PW>(p, PH(sy) - PH(0)),
            divx<PW>(p, PH(0) - PH(-sy)), divx<PW>(p, PH(-sy) - PH(-2 * sy)));
  if (k >= 3 && k <= p.kmax - 2) {
    E = weno5(divz<PW>(p, PH(-2 * sz) - PH(-3 * sz)), divz<PW>(p, PH(-sz) - PH(-2 * sz)), divz<PW>(p, PH(0) - PH(-sz)),
              divz<PW>(p, PH(sz) - PH(0)), divz<PW>(p, PH(2 * sz) - PH(sz)));
    F = weno5(divz<PW>(p, PH(3 * sz) - PH(2 * sz)), divz<PW>(p, PH(2 * sz) - PH(sz)), divz<PW>(p, PH(sz) - PH(0)),
              divz<PW>(p, PH(0) - PH(-sz)), divz<PW>(p, PH(-sz) - PH(-2 * sz)));
  } else {
    E = divz<PW>(p, PH(0) - PH(-sz));
    F = divz<PW>(p, PH(sz) - PH(0));
  }
#undef PH
  const T s = reinit_sgn(p, orig[c]);
  T dydx, dydy, dydz;
  if (p.TwoD) {
    dydx = TC(0.);
  } else {
    if ((B * s < TC(0.)) && ((A + B) * s < TC(0.))) dydx = B;
    else if ((A * s > TC(0.)) && ((A + B) * s > TC(0.))) dydx = A;
    else dydx = TC(0.5) * (A + B);
  }
  if ((D * s < TC(0.)) && ((C + D) * s < TC(0.))) dydy = D;
  else if ((C * s > TC(0.)) && ((C + D) * s > TC(0.))) dydy = C;
  else dydy = TC(0.5) * (C + D);
  if ((F * s < TC(0.)) && ((E + F) * s < TC(0.))) dydz = F;
  else if ((E * s > TC(0.)) && ((E + F) * s > TC(0.))) dydz = E;
  else dydz = TC(0.5) * (E + F);
  return s * (TC(1.) - sqrt((dydx * dydx + dydy * dydy) + dydz * dydz));
}

// one SSP-RK3 stage value of ls_reinit (levelset.f90:800-810)
template <int PW, typename T>
__device__ __forceinline__ T reinit_val(const Params& p, int stage, const T* __restrict__ phi0,
                                        const T* __restrict__ phis, const T* __restrict__ orig, T dtau, int I, int J,
                                        int k) {
  const long long n = idxL(p, I, J, k);
  const T rhs = (k >= 1 && k <= p.kmax) ? reinit_rhs<PW>(p, phis, orig, I, J, k) : TC(0.);
  if (stage == 1) return phi0[n] + dtau * rhs;
  if (stage == 2) return TC(3. / 4.) * phi0[n] + TC(1. / 4.) * (phis[n] + dtau * rhs);
  return TC(1. / 3.) * phi0[n] + TC(2. / 3.) * (phis[n] + dtau * rhs);
}

// One SSP-RK3 stage of ls_reinit over the tasks' regions; stage 3 folds
// max|phi_new - phi_0| into the drop's residual.  out may equal phi0.
template <typename T, int PW>
__global__ void __launch_bounds__(NT, (sizeof(T) == 4 ? 4 : 3)) k_reinit_stage(Params p, const __grid_constant__ LsBatch B, int stage,
                                                        double dtau_, ReinitState* __restrict__ rs) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const T* phi0 = cT<T>(t.phi0);
  T* out = mT<T>(t.out);
  if (rs[t.l].done) {
    // an iteration after convergence is the identity (levelset.f90:833-835)
    if (stage == 3 && c.ok && t.out != t.phi0)
      for (int k = c.ka; k <= c.kb; ++k) putL(p, out, c.i, c.j, k, phi0[idxL(p, c.i, c.j, k)]);
    return;
  }
  const T dtau = TC(dtau_);
  double r = 0.;
  if (c.ok) {
    const T* phis = cT<T>(t.phis);
    const T* orig = cT<T>(t.orig);
    const int i = c.i, j = c.j;
    T v1 = TC(0.), v2 = TC(0.), vkm = TC(0.), vk = TC(0.);
    bool wall0 = false;
    for (int k = c.ka; k <= c.kb; ++k) {
      if (!computed(c, t.r, k)) {
        putL(p, out, i, j, k, (k < 0 || k > p.k1) ? TC(t.bgg) : TC(t.bg));
        continue;
      }
      if (k == 0) {
        wall0 = true;
        continue;
      }
      T val;
      if (k == p.k1) {
        val = TC(2.) * vk - vkm;
      } else {
        val = reinit_val<PW>(p, stage, phi0, phis, orig, dtau, i, j, k);
        if (k == 1) v1 = val;
        if (k == 2) v2 = val;
        if (k == p.kmax - 1) vkm = val;
        if (k == p.kmax) vk = val;
      }
      if (stage == 3) r = fmax(r, (double)fabs(val - phi0[idxL(p, i, j, k)]));
      putL(p, out, i, j, k, val);
      if (k == 2 && wall0) {
        const T v0 = TC(2.) * v1 - v2;
        if (stage == 3) r = fmax(r, (double)fabs(v0 - phi0[idxL(p, i, j, 0)]));
        putL(p, out, i, j, 0, v0);
      }
    }
  }
  if (stage == 3) {
    const double bm = block_max<double, NT>(r);
    if (flat_tid() == 0) atomic_max_nonneg(&rs[t.l].residual, bm);
  }
}

__global__ void k_reinit_reset(const __grid_constant__ LsBatch B, int maxiter, ReinitState* __restrict__ rs) {
  for (int q = threadIdx.x; q < B.n; q += blockDim.x) {
    ReinitState& s = rs[B.t[q].l];
    s.residual = 0.;
    s.last = 0.;
    s.done = 0;
    s.iters = maxiter;
  }
}
// end of iteration `it`: far is the change of the far-field cells outside
// the drop's region (0 when none); the last drop's state is also published
// as the scalars of the last ls_reinit call
__global__ void k_reinit_check(const __grid_constant__ LsBatch B, int it, int maxiter, double thr,
                               ReinitState* __restrict__ rs, DevScalars* __restrict__ dsc, int last_drop) {
  for (int q = threadIdx.x; q < B.n; q += blockDim.x) {
    const int l = B.t[q].l;
    ReinitState& s = rs[l];
    if (!s.done) {
      double r = s.residual;
      if (B.t[q].far > r) r = B.t[q].far;
      s.last = r;
      s.residual = 0.;
      if (r < thr) {
        s.done = 1;
        s.iters = it;
      } else {
        s.iters = maxiter;
      }
    }
    if (l == last_drop) {
      dsc->residual = s.last;
      dsc->reinit_iters = s.iters;
      dsc->reinit_done = s.done;
    }
  }
}

// --------------------------------------------------------- Heaviside
template <typename T>
__device__ __forceinline__ T heav_trig(const Params& p, T phi, T eps) {
  if (phi < -eps) return TC(0.);
  if (phi < eps) return (TC(.5) + TC(.5) * phi / eps) + TC(.5) / TC(p.pi) * sin(TC(p.pi) * phi / eps);
  return TC(1.);
}
template <typename T>
__device__ __forceinline__ T dirac_trig(const Params& p, T phi, T eps) {
  if (phi < -eps) return TC(0.);
  if (phi < eps) return TC(.5) / eps + TC(.5) / eps * cos(TC(p.pi) * phi / eps);
  return TC(0.);
}

// disp_cg and disp_speed (write_vtk.f90:438-566) of one drop: over the
// interior cells with phi <= 1.5 dz, the count, the sums of the cell-centre
// coordinates (i - 1/2)/dxi, ... and of ucc dx dy dz (1 - H), ... (H the
// 'trig' Heaviside of the drop).  Warp w of the grid takes the rows (j,k)
// w, w + W, ...; per-block partials part[7 * block + q] in a fixed order.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_disp(Params p, const T* __restrict__ phi,
                                                      const T* __restrict__ ucc, const T* __restrict__ vcc,
                                                      const T* __restrict__ wcc, double* __restrict__ part) {
  double s[7] = {0., 0., 0., 0., 0., 0., 0.};
  const int rows = p.jmax * p.kmax;
  const int W = (int)((gridDim.x * kRedThreads) >> 5);
  const int lane = threadIdx.x & 31;
  const T lim = TC(1.5 * p.dz), eps = TC(1.5 * p.dz);
  for (int r = (int)((blockIdx.x * kRedThreads + threadIdx.x) >> 5); r < rows; r += W) {
    const int j = 1 + r % p.jmax, k = 1 + r / p.jmax;
    const double cy = (j - 0.5) / p.dyi, cz = (k - 0.5) / p.dzi;
    for (int i = 1 + lane; i <= p.imax; i += 32) {
      const T f = phi[idxL(p, i, j, k)];
      if (f <= lim) {
        const long long q = idxI(p, i, j, k);
        const double g = 1. - (double)heav_trig(p, f, eps);
        s[0] += 1.;
        s[1] += (i - 0.5) / p.dxi;
        s[2] += cy;
        s[3] += cz;
        s[4] += ((((double)ucc[q] * p.dx) * p.dy) * p.dz) * g;
        s[5] += ((((double)vcc[q] * p.dx) * p.dy) * p.dz) * g;
        s[6] += ((((double)wcc[q] * p.dx) * p.dy) * p.dz) * g;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    const double b = block_sum<double, kRedThreads>(s[q]);
    if (threadIdx.x == 0) part[7 * blockIdx.x + q] = b;
  }
}
__global__ void __launch_bounds__(kRedThreads) k_disp_final(const double* __restrict__ part, int nblk,
                                                            double* __restrict__ out) {
#pragma unroll 1
  for (int q = 0; q < 7; ++q) {
    double s = 0.;
    for (int b = threadIdx.x; b < nblk; b += kRedThreads) s += part[7 * b + q];
    s = block_sum<double, kRedThreads>(s);
    if (threadIdx.x == 0) out[q] = s;
  }
}

// jiemian = min(jiemian, H_l) over the tasks' computed cells (shape-C
// regions) and per-tile sums of H_l over their interior cells
// (misc.f90:110-141), the sums in FP64.  jiemian starts at 1, the
// far-field value of H, so only cells with H < 1 are touched; min is
// order-free, so drops may share cells.  One chunk per tile:
// part[l*cap + tile] is deterministic.
// For v >= +0 the signed-integer order of the bit patterns is the numeric
// order against every non-negative value, and every negative value (sign
// bit set) compares below it, as it does numerically: one atomicMin that
// returns nothing (the thread does not wait for it).  A negative v (H is
// negative only by rounding, ~1e-17) takes the compare-and-swap loop.
__device__ __forceinline__ void min_into(double* a, double v) {
  if (!(v < 0.)) {
    atomicMin(reinterpret_cast<long long*>(a), __double_as_longlong(v));
    return;
  }
  unsigned long long* q = reinterpret_cast<unsigned long long*>(a);
  unsigned long long old = *q;
  while (v < __longlong_as_double((long long)old)) {
    const unsigned long long prev = atomicCAS(q, old, (unsigned long long)__double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}
__device__ __forceinline__ void min_into(float* a, float v) {
  if (!(v < 0.f)) {
    atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
    return;
  }
  unsigned int* q = reinterpret_cast<unsigned int*>(a);
  unsigned int old = *q;
  while (v < __uint_as_float(old)) {
    const unsigned int prev = atomicCAS(q, old, __float_as_uint(v));
    if (prev == old) break;
    old = prev;
  }
}
template <typename T>
__global__ void __launch_bounds__(NT, 4) k_heaviside(Params p, const __grid_constant__ LsBatch B,
                                                  T* __restrict__ jiemian, XSum* __restrict__ part, int cap) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const T eps = TC(1.5 * p.dz);
  const T* __restrict__ phi = cT<T>(t.phi0);
  XSum s;
  xs_zero(s);
  if (c.ok && c.cxy) {
    const int i = c.i, j = c.j;
    const int ii = image_of<1>(i, p.imax), jj = image_of<1>(j, p.jmax);
    const int ka = max(c.ka, t.r.cz0), kb = min(c.kb, t.r.cz1);
    const long long sz = (long long)p.nLx * p.nLy;
    // eight rows' phi in flight before their minima and sums (same order)
    for (int k0 = ka; k0 <= kb; k0 += 8) {
      T f[8];
      const long long c0 = idxL(p, i, j, k0);
#pragma unroll
      for (int u = 0; u < 8; ++u) f[u] = (k0 + u <= kb) ? phi[c0 + u * sz] : TC(1.);
#pragma unroll
      for (int u = 0; u < 8; ++u) {  // rows past kb skipped without a break, so f stays in registers
        const int k = k0 + u;
        if (k <= kb) {
          const T H = heav_trig(p, f[u], eps);
          if (H < TC(1.)) {
            min_into(jiemian + idxC(p, i, j, k), H);
            if (ii != INT_MIN) min_into(jiemian + idxC(p, ii, j, k), H);
            if (jj != INT_MIN) {
              min_into(jiemian + idxC(p, i, jj, k), H);
              if (ii != INT_MIN) min_into(jiemian + idxC(p, ii, jj, k), H);
            }
          }
          if (k >= 1 && k <= p.kmax) xs_add(s, (double)H);
        }
      }
    }
  }
  const XSum bs = block_xsum<NT>(s);
  // one partial per (column tile, z chunk) of the task
  if (flat_tid() == 0) part[(long long)t.l * cap + c.tile + (long long)t.tx * t.ty * c.ch] = bs;
}

// volume(l) and rho_avr from the per-tile sums (misc.f90:139-173);
// outside[l] interior cells of drop l lie in its far field, where H = 1
struct PerDrop {
  double v[kMaxDropsParam];
  int n[kMaxDropsParam];
};
// One warp per drop: its lanes merge every 32nd partial, the lanes' sums
// (limbs below 2^48 after each merge) add limb by limb across the warp
// (below 2^53), and lane 0 rounds the exact total once.
__global__ void k_volumes(Params p, const XSum* __restrict__ part, int cap, PerDrop pd, int uniform, int nb_all,
                          double* __restrict__ vol, DevScalars* __restrict__ dsc) {
  const double N = (1. * p.imax * p.jmax) * p.kmax;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int l = warp; l < p.L; l += nw) {
    const int nb = uniform ? nb_all : pd.n[l];
    XSum s;
    xs_zero(s);
    for (int b = lane; b < nb; b += 32) xs_merge(s, part[(long long)l * cap + b]);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      for (int d = 16; d > 0; d >>= 1) s.L[q] += __shfl_down_sync(0xffffffffu, s.L[q], d);
    if (lane == 0) {
      xs_norm(s);
      if (!uniform) xs_add_count(s, (long long)pd.v[l]);
      vol[l] = 1. - xs_value(s) / N;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sv = 0.;
    for (int l = 0; l < p.L; ++l) sv += vol[l];
    dsc->rho_avr = p.rho1 * (1. - sv) + p.rho2 * sv;
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k_fill(T* __restrict__ a, long long n, double v) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    a[q] = TC(v);
}

// miu, rho (shape C) and the face densities (misc.f90:121-172)
template <typename T>
__global__ void __launch_bounds__(NT) k_materials_final(Params p, const T* __restrict__ jiemian, T* __restrict__ miu,
                                                        T* __restrict__ rho, T* __restrict__ rho_u,
                                                        T* __restrict__ rho_v, T* __restrict__ rho_w) {
  const int r0[3] = {0, 0, 0}, r1[3] = {p.i1, p.j1, p.k1};
  int i, j, k;
  if (!cell3(r0, r1, i, j, k)) return;
  const long long n = idxC(p, i, j, k);
  const T rho1 = TC(p.rho1), rho2 = TC(p.rho2);
  const T J0 = jiemian[n];
  miu[n] = TC(p.miu1) * J0 + TC(p.miu2) * (TC(1.) - J0);
  const T r0v = rho1 * J0 + rho2 * (TC(1.) - J0);
  rho[n] = r0v;
  if (interior(p, i, j, k)) {
    const long long q = idxI(p, i, j, k);
    if (p.rho1 == p.rho2) {
      rho_u[q] = rho1; rho_v[q] = rho1; rho_w[q] = rho1;
    } else {
      const T Jx = jiemian[n + 1], Jy = jiemian[n + p.nCx], Jz = jiemian[n + (long long)p.nCx * p.nCy];
      const T rx = rho1 * Jx + rho2 * (TC(1.) - Jx);
      const T ry = rho1 * Jy + rho2 * (TC(1.) - Jy);
      const T rz = rho1 * Jz + rho2 * (TC(1.) - Jz);
      rho_u[q] = (r0v + rx) / TC(2.);
      rho_v[q] = (r0v + ry) / TC(2.);
      rho_w[q] = (r0v + rz) / TC(2.);
    }
  }
}

// k_materials_final over two rows per thread (k0 = 2 blockIdx.z and k0 + 1):
// both rows' jiemian values are read before any store, so a thread has its
// two cells' loads in flight at once; the same expressions per cell
template <typename T>
__device__ __forceinline__ void materials_cell(const Params& p, long long n, long long q, bool in, T J0, T Jx, T Jy,
                                               T Jz, T* __restrict__ miu, T* __restrict__ rho, T* __restrict__ rho_u,
                                               T* __restrict__ rho_v, T* __restrict__ rho_w) {
  const T rho1 = TC(p.rho1), rho2 = TC(p.rho2);
  miu[n] = TC(p.miu1) * J0 + TC(p.miu2) * (TC(1.) - J0);
  const T r0v = rho1 * J0 + rho2 * (TC(1.) - J0);
  rho[n] = r0v;
  if (!in) return;
  if (p.rho1 == p.rho2) {
    rho_u[q] = rho1; rho_v[q] = rho1; rho_w[q] = rho1;
  } else {
    const T rx = rho1 * Jx + rho2 * (TC(1.) - Jx);
    const T ry = rho1 * Jy + rho2 * (TC(1.) - Jy);
    const T rz = rho1 * Jz + rho2 * (TC(1.) - Jz);
    rho_u[q] = (r0v + rx) / TC(2.);
    rho_v[q] = (r0v + ry) / TC(2.);
    rho_w[q] = (r0v + rz) / TC(2.);
  }
}
template <typename T>
__global__ void __launch_bounds__(NT) k_materials_rows2(Params p, const T* __restrict__ jiemian, T* __restrict__ miu,
                                                        T* __restrict__ rho, T* __restrict__ rho_u,
                                                        T* __restrict__ rho_v, T* __restrict__ rho_w) {
  const int i = (int)(blockIdx.x * BX + threadIdx.x), j = (int)(blockIdx.y * BY + threadIdx.y);
  const int k0 = 2 * (int)blockIdx.z;
  if (i > p.i1 || j > p.j1) return;
  const bool two = k0 + 1 <= p.k1;
  const long long sz = (long long)p.nCx * p.nCy;
  const long long n0 = idxC(p, i, j, k0), n1 = n0 + sz;
  const bool in0 = interior(p, i, j, k0), in1 = two && interior(p, i, j, k0 + 1);
  const T Ja = jiemian[n0];
  const T Jb = two ? jiemian[n1] : TC(0.);
  T Jxa = TC(0.), Jya = TC(0.), Jxb = TC(0.), Jyb = TC(0.), Jzb = TC(0.);
  if (in0) {
    Jxa = jiemian[n0 + 1];
    Jya = jiemian[n0 + p.nCx];
  }
  if (in1) {
    Jxb = jiemian[n1 + 1];
    Jyb = jiemian[n1 + p.nCx];
    Jzb = jiemian[n1 + sz];
  }
  materials_cell<T>(p, n0, in0 ? idxI(p, i, j, k0) : 0, in0, Ja, Jxa, Jya, Jb, miu, rho, rho_u, rho_v, rho_w);
  if (two)
    materials_cell<T>(p, n1, in1 ? idxI(p, i, j, k0 + 1) : 0, in1, Jb, Jxb, Jyb, Jzb, miu, rho, rho_u, rho_v, rho_w);
}

// ------------------------------------------------------------ inflation
// dheav with boundp semantics over the task's shape-C region (one task),
// the far-field value 1 on its apron, and per-tile area/volume sums (FP64)
// over its interior computed cells (levelset.f90:493-507, 525)
template <typename T>
__global__ void __launch_bounds__(NT) k_inflate_sums(Params p, const __grid_constant__ LsBatch B,
                                                     const T* __restrict__ kappa, const T* __restrict__ nrm_m,
                                                     T* __restrict__ dheav, double* __restrict__ part_area,
                                                     XSum* __restrict__ part_heav) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const T s1 = TC(1.5 * p.dz);
  const T* phi = cT<T>(t.phi0);
  double sa = 0.;
  XSum sh;
  xs_zero(sh);
  if (c.ok) {
    const int i = c.i, j = c.j;
    for (int k = c.ka; k <= c.kb; ++k) {
      if (!computed(c, t.r, k)) {
        putC(p, dheav, i, j, k, TC(1.));
        continue;
      }
      const int K = k == 0 ? 1 : (k == p.k1 ? p.kmax : k);
      putC(p, dheav, i, j, k, heav_trig(p, phi[idxL(p, i, j, K)], s1));
      if (k >= 1 && k <= p.kmax) {
        const T ph = phi[idxL(p, i, j, k)];
        const T H = heav_trig(p, ph, s1);
        const T del = dirac_trig(p, ph, s1);
        const T m = nrm_m[idxI(p, i, j, k)];
        sa += (double)(p.ispeed_curv ? (del * kappa[idxC(p, i, j, k)]) * m : del * m);
        xs_add(sh, (double)H);
      }
    }
  }
  const double ba = block_sum<double, NT>(sa);
  const XSum bh = block_xsum<NT>(sh);
  if (flat_tid() == 0) {
    part_area[c.tile] = ba;
    part_heav[c.tile] = bh;
  }
}

__global__ void k_inflate_final(Params p, const double* __restrict__ part_area,
                                const XSum* __restrict__ part_heav, int nblk, int l, double istep_dt,
                                double outside, double* __restrict__ vol, const double* __restrict__ vol0,
                                double* __restrict__ maxchk, DevScalars* __restrict__ dsc) {
  if (threadIdx.x != 0) return;
  double sa = 0.;
  XSum hs;
  xs_zero(hs);
  for (int b = 0; b < nblk; ++b) {
    sa += part_area[b];
    xs_merge(hs, part_heav[b]);
  }
  xs_add_count(hs, (long long)outside);
  const double sh = xs_value(hs);
  double area = sa * p.dx * p.dy * p.dz;
  if (p.TwoD) area = area / p.lx;
  const double volume = 1. - sh / ((1. * p.imax * p.jmax) * p.kmax);
  vol[l] = volume;
  double loss_rate = p.lx * p.ly * p.lz * (volume - vol0[l]) / istep_dt;
  if (p.TwoD) loss_rate = loss_rate / p.lx;
  const double temp = loss_rate / area;
  dsc->inflate_temp = temp;
  dsc->area = area;
  dsc->heav_sum = sh;
  maxchk[l] = temp / (1.5 * p.dz);
}

// ------------------------------------------------ gain-one mass correction
// icls_config.mass_gain_one (no counterpart in the reference).  The
// reference's inflation moves the interface by about K/inflate_step times
// the volume error it measured (K ~ 0.66/s1 in grid units), so with the
// option the inflated level set phi1 is blended with the one before it,
// phi = phi0 + g (phi1 - phi0), g = (V0 - V)/(V1 - V) from the exact
// volumes before (V) and after (V1) the inflation: the blend removes the
// measured error to first order in the (small) displacement.

// t.out = t.phi0 on the task's written cells (rows of the chunk, images)
template <typename T>
__global__ void __launch_bounds__(NT) k_region_copy(Params p, const __grid_constant__ LsBatch B) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok) return;
  const T* __restrict__ src = cT<T>(t.phi0);
  T* __restrict__ dst = mT<T>(t.out);
  for (int k = c.ka; k <= c.kb; ++k) putL(p, dst, c.i, c.j, k, src[idxL(p, c.i, c.j, k)]);
}

// per-tile exact sums of H(phi1) over the task's computed interior cells
template <typename T>
__global__ void __launch_bounds__(NT) k_region_heav(Params p, const __grid_constant__ LsBatch B,
                                                    XSum* __restrict__ part) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  const T s1 = TC(1.5 * p.dz);
  const T* __restrict__ phi = cT<T>(t.phi0);
  XSum sh;
  xs_zero(sh);
  if (c.ok)
    for (int k = max(c.ka, 1); k <= min(c.kb, p.kmax); ++k)
      if (computed(c, t.r, k)) xs_add(sh, (double)heav_trig(p, phi[idxL(p, c.i, c.j, k)], s1));
  const XSum bh = block_xsum<NT>(sh);
  if (flat_tid() == 0) part[c.tile] = bh;
}

// g = (V0 - V)/(V1 - V), V1 from the tiles and the far-field count
__global__ void k_gain_final(Params p, const XSum* __restrict__ part, int nblk, int l, double outside,
                             const double* __restrict__ vol, const double* __restrict__ vol0,
                             DevScalars* __restrict__ dsc) {
  if (threadIdx.x != 0) return;
  XSum hs;
  xs_zero(hs);
  for (int b = 0; b < nblk; ++b) xs_merge(hs, part[b]);
  xs_add_count(hs, (long long)outside);
  const double v1 = 1. - xs_value(hs) / ((1. * p.imax * p.jmax) * p.kmax);
  const double d = v1 - vol[l];
  dsc->inflate_gain = d != 0. ? (vol0[l] - vol[l]) / d : 0.;
}

// the volume of drop l now, from the tiles and the far-field count
__global__ void k_volume_now(Params p, const XSum* __restrict__ part, int nblk, int l, double outside,
                             double* __restrict__ vnow) {
  if (threadIdx.x != 0) return;
  XSum hs;
  xs_zero(hs);
  for (int b = 0; b < nblk; ++b) xs_merge(hs, part[b]);
  xs_add_count(hs, (long long)outside);
  vnow[l] = 1. - xs_value(hs) / ((1. * p.imax * p.jmax) * p.kmax);
}

// t.out (phi1, in place) = phi0 + g (phi1 - phi0) on the written cells
template <typename T>
__global__ void __launch_bounds__(NT) k_region_blend(Params p, const __grid_constant__ LsBatch B,
                                                     const DevScalars* __restrict__ dsc) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok) return;
  const double g = dsc->inflate_gain;
  const T* __restrict__ p0 = cT<T>(t.phi0);
  T* __restrict__ p1 = mT<T>(t.out);
  for (int k = c.ka; k <= c.kb; ++k) {
    const long long n = idxL(p, c.i, c.j, k);
    const double a0 = (double)p0[n];
    putL(p, p1, c.i, c.j, k, TC(a0 + g * ((double)p1[n] - a0)));
  }
}

// u_lc, v_lc, w_lc of levelset.f90:527-548, with u_l,v_l,w_l of 530-532
// after bounduvw evaluated on the fly; computed interior cells of r
template <typename T>
__device__ __forceinline__ T infl_face(const Params& p, const T* __restrict__ dheav, T temp, int axis, int i, int j,
                                       int k) {
  const long long n = idxC(p, i, j, k);
  if (axis == 0) return -divx(p, temp * (dheav[n + 1] - dheav[n]));
  if (axis == 1) return -divy(p, temp * (dheav[n + p.nCx] - dheav[n]));
  return -divz(p, temp * (dheav[n + (long long)p.nCx * p.nCy] - dheav[n]));
}
// v_l(i,0,k) and v_l(i,jmax,k) with the y walls of boundp(dheav) and
// bounduvw(u_l,v_l,w_l) (levelset.f90:466-478, bound.f90:81-282) for
// BC_in_y = Walls, InOut, OutOut: v_l = 0 on a wall, v_inflow at the inlet,
// the OutOut extrapolation at y = 0, and dheav(i,j1,k) = -dheav(i,jmax,k) at
// an outflow end
template <typename T>
__device__ __forceinline__ T infl_v_front(const Params& p, const T* __restrict__ dheav, T temp, int i, int k,
                                          const double* __restrict__ vin) {
  if (p.bcy == ICLS_BCY_WALLS) return TC(0.);
  if (p.bcy == ICLS_BCY_INOUT) return TC(vin[i + (long long)(p.i1 + 1) * k]);
  const T wl_1 = (k == p.kmax) ? TC(0.) : infl_face(p, dheav, temp, 2, i, 1, k);
  const T wl_0 = (k == 1) ? TC(0.) : infl_face(p, dheav, temp, 2, i, 1, k - 1);
  return infl_face(p, dheav, temp, 1, i, 1, k) + TC(p.dy / p.dz) * (wl_1 - wl_0);
}
template <typename T>
__device__ __forceinline__ T infl_v_back(const Params& p, const T* __restrict__ dheav, T temp, int i, int k) {
  if (p.bcy == ICLS_BCY_WALLS) return TC(0.);
  const T h = dheav[idxC(p, i, p.jmax, k)];
  return -divy(p, temp * (-h - h));
}
template <typename T>
__global__ void __launch_bounds__(NT) k_inflate_vel(Params p, const __grid_constant__ LsBatch B,
                                                    const T* __restrict__ dheav, const T* __restrict__ kappa,
                                                    const DevScalars* __restrict__ dsc, T* __restrict__ ulc,
                                                    T* __restrict__ vlc, T* __restrict__ wlc,
                                                    const double* __restrict__ vin) {
  const int ti = task_of(B);
  const LsTask& t = B.t[ti];
  const Col c = col_of(p, t, (int)blockIdx.x - B.start[ti]);
  if (!c.ok || !c.cxy) return;
  const int i = c.i, j = c.j;
  const T temp = TC(dsc->inflate_temp);
  for (int k = max(c.ka, max(t.r.cz0, 1)); k <= min(c.kb, min(t.r.cz1, p.kmax)); ++k) {
    const long long q = idxI(p, i, j, k);
    const T ul_m = infl_face(p, dheav, temp, 0, wrapx(p, i - 1), j, k);
    const T ul_0 = infl_face(p, dheav, temp, 0, i, j, k);
    T vl_m, vl_0;
    if (p.bcy == ICLS_BCY_PERIODIC || (j != 1 && j != p.jmax)) {
      vl_m = infl_face(p, dheav, temp, 1, i, wrapy(p, j - 1), k);
      vl_0 = infl_face(p, dheav, temp, 1, i, j, k);
    } else {
      vl_m = j == 1 ? infl_v_front(p, dheav, temp, i, k, vin) : infl_face(p, dheav, temp, 1, i, j - 1, k);
      vl_0 = j == p.jmax ? infl_v_back(p, dheav, temp, i, k) : infl_face(p, dheav, temp, 1, i, j, k);
    }
    const T wl_m = (k == 1) ? TC(0.) : infl_face(p, dheav, temp, 2, i, j, k - 1);
    const T wl_0 = (k == p.kmax) ? TC(0.) : infl_face(p, dheav, temp, 2, i, j, k);
    T a = (ul_m + ul_0) / TC(2.), b = (vl_m + vl_0) / TC(2.), cc = (wl_m + wl_0) / TC(2.);
    if (p.ispeed_curv) {
      const T kp = kappa[idxC(p, i, j, k)];
      a = a * kp; b = b * kp; cc = cc * kp;
    }
    ulc[q] = a; vlc[q] = b; wlc[q] = cc;
  }
}

// boundmls, extrap='line' (bound.f90:518-~657): three wall layers by
// repeated linear extrapolation from the interior column, then the periodic
// copies.  Reads only interior cells, writes only the others.
template <typename T>
__global__ void __launch_bounds__(NT) k_boundmls(Params p, T* __restrict__ y) {
  const int r0[3] = {-2, -2, -2}, r1[3] = {p.i1 + 2, p.j1 + 2, p.k1 + 2};
  int i, j, k;
  if (!cell3(r0, r1, i, j, k)) return;
  const long long n = idxL(p, i, j, k);
  const int I = wrapx(p, i), J = wrapy(p, j);
  if (k >= 1 && k <= p.kmax) {
    if (I != i || J != j) y[n] = y[idxL(p, I, J, k)];
    return;
  }
  if (k <= 0) {
    const T y1 = y[idxL(p, I, J, 1)], y2 = y[idxL(p, I, J, 2)];
    const T y0 = TC(2.) * y1 - y2;
    const T ym1 = TC(2.) * y0 - y1;
    const T ym2 = TC(2.) * ym1 - y0;
    y[n] = (k == 0) ? y0 : (k == -1 ? ym1 : ym2);
  } else {
    const T yk = y[idxL(p, I, J, p.kmax)], ykm = y[idxL(p, I, J, p.kmax - 1)];
    const T y0 = TC(2.) * yk - ykm;
    const T yp1 = TC(2.) * y0 - yk;
    const T yp2 = TC(2.) * yp1 - y0;
    y[n] = (k == p.k1) ? y0 : (k == p.k1 + 1 ? yp1 : yp2);
  }
}

// far-field value into every cell outside the written cells of r (makes a
// drop's stored array valid everywhere, e.g. before a download)
template <typename T>
__global__ void __launch_bounds__(NT) k_materialize(Params p, Region r, double bg, double bgg, T* __restrict__ y) {
  const int r0[3] = {-2, -2, -2}, r1[3] = {p.i1 + 2, p.j1 + 2, p.k1 + 2};
  int i, j, k;
  if (!cell3(r0, r1, i, j, k)) return;
  if (!in_written(p, r, i, j, k)) y[idxL(p, i, j, k)] = (k < 0 || k > p.k1) ? TC(bgg) : TC(bg);
}

template <typename T>
__global__ void k_copy(T* __restrict__ dst, const T* __restrict__ src, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = src[q];
}

// field conversions of the precision form (upload / download)
__global__ void k_to_float(float* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = (float)src[q];
}
__global__ void k_to_double(double* __restrict__ dst, const float* __restrict__ src, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = (double)src[q];
}

#undef TC

}  // namespace

dim3 grid_of(const int* r0, const int* r1) {
  const int nx = r1[0] - r0[0] + 1, ny = r1[1] - r0[1] + 1, nz = r1[2] - r0[2] + 1;
  return dim3((unsigned)((nx + BX - 1) / BX), (unsigned)((ny + BY - 1) / BY), (unsigned)nz);
}

namespace {
int wrap1(int v, int n) {
  v = (v - 1) % n;
  if (v < 0) v += n;
  return v + 1;
}
}  // namespace

Region full_region(const Params& P) {
  Region r;
  r.xa = 1; r.xn = P.imax; r.cx0 = 0; r.cx1 = P.imax - 1;
  r.ya = 1; r.yn = P.jmax; r.cy0 = 0; r.cy1 = P.jmax - 1;
  r.z0 = r.cz0 = -2;
  r.z1 = r.cz1 = P.k1 + 2;
  return r;
}

bool region_full(const Params& P, const Region& r) {
  return r.xn == P.imax && r.cx0 == 0 && r.cx1 == P.imax - 1 && r.yn == P.jmax && r.cy0 == 0 &&
         r.cy1 == P.jmax - 1 && r.cz0 <= -2 && r.cz1 >= P.k1 + 2;
}

// the shape-C region of a level-set region: the same computed columns with
// an apron of `ap` columns; full z becomes rows 0..k1
Region c_region(const Params& P, const Region& r, int ap) {
  Region q;
  auto axis = [&](int xa, int xn, int c0, int c1, int n, int& qa, int& qn, int& q0, int& q1) {
    if (xn == n && c0 == 0 && c1 == n - 1) {
      qa = 1; qn = n; q0 = 0; q1 = n - 1;
      return;
    }
    const int a = wrap1(xa + c0, n), len = c1 - c0 + 1;
    qa = wrap1(a - ap, n);
    qn = len + 2 * ap;
    q0 = ap;
    q1 = ap + len - 1;
  };
  axis(r.xa, r.xn, r.cx0, r.cx1, P.imax, q.xa, q.xn, q.cx0, q.cx1);
  axis(r.ya, r.yn, r.cy0, r.cy1, P.jmax, q.ya, q.yn, q.cy0, q.cy1);
  if (r.cz0 <= -2 && r.cz1 >= P.k1 + 2) {
    q.z0 = q.cz0 = 0;
    q.z1 = q.cz1 = P.k1;
  } else {
    q.cz0 = r.cz0;
    q.cz1 = r.cz1;
    q.z0 = std::max(0, r.cz0 - ap);
    q.z1 = std::min(P.k1, r.cz1 + ap);
  }
  return q;
}

// tiles, z chunks (kc rows each, the last one longer; kc <= 0: one chunk)
// and block offsets of a batch; flat tiles of 256 consecutive columns
// (col_of), or TBX x TBY tiles for the kernels that stage a 2-D tile
void set_tiles(LsBatch& b, int kc, bool flat) {
  int s = 0;
  for (int q = 0; q < b.n; ++q) {
    LsTask& t = b.t[q];
    t.flat = flat ? 1 : 0;
    if (flat) {
      t.tx = (t.r.xn * t.r.yn + TBX * TBY - 1) / (TBX * TBY);
      t.ty = 1;
    } else {
      t.tx = (t.r.xn + TBX - 1) / TBX;
      t.ty = (t.r.yn + TBY - 1) / TBY;
    }
    const int nz = t.r.z1 - t.r.z0 + 1;
    if (kc <= 0 || kc >= nz) {
      t.nch = 1;
      t.kc = nz;
    } else {
      t.nch = nz / kc;
      t.kc = kc;
    }
    b.start[q] = s;
    s += t.tx * t.ty * t.nch;
  }
  b.start[b.n] = s;
}

// ================================================================ launchers
// Each launcher picks the field type of the context's form.
#define BY_FORM(c, call_f32, call_f64) \
  do {                                  \
    if ((c).P.f32) {                    \
      call_f32;                         \
    } else {                            \
      call_f64;                         \
    }                                   \
  } while (0)

void launch_tube(Ctx& c, const LsBatch& flat) {
  if (flat.n == 0) return;
  Scope sc_(c.prof, c.s, "tube", 1);
  // k_tube stages a TBX x TBY tile with its halo in shared memory: the same
  // tasks on 2-D tiles, in z chunks of kTubeRows rows (its register window
  // along z favours longer chunks than the stage kernels': 16 rows measured
  // 0.135 -> 0.128 ms FP32, 0.206 -> 0.188 ms FP64 against 8)
  constexpr int kTubeRows = 16;
  LsBatch b = flat;
  int s = 0;
  for (int q = 0; q < b.n; ++q) {
    LsTask& t = b.t[q];
    t.flat = 0;
    t.tx = (t.r.xn + TBX - 1) / TBX;
    t.ty = (t.r.yn + TBY - 1) / TBY;
    const int nz = t.r.z1 - t.r.z0 + 1;
    if (kTubeRows >= nz) {
      t.nch = 1;
      t.kc = nz;
    } else {
      t.nch = nz / kTubeRows;
      t.kc = kTubeRows;
    }
    b.start[q] = s;
    s += t.tx * t.ty * t.nch;
  }
  b.start[b.n] = s;
  int* lo = c.d_bbox;
  int* hi = c.d_bbox + 5 * c.P.L;
  BY_FORM(c, (k_tube<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.d_nbcnt, lo, hi)),
          (k_tube<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.d_nbcnt, lo, hi)));
}

void launch_band_extents(Ctx& c, int l) {
  Scope sc_(c.prof, c.s, "band_extents", 1);
  int* lo = c.d_bbox;
  int* hi = c.d_bbox + 5 * c.P.L;
  const unsigned g = (unsigned)(((long long)c.P.imax * c.P.jmax + NT - 1) / NT);
  BY_FORM(c, (k_band_extents<float><<<g, NT, 0, c.s>>>(c.P, reinterpret_cast<const float*>(c.lv[l]), l, lo, hi)),
          (k_band_extents<double><<<g, NT, 0, c.s>>>(c.P, c.lv[l], l, lo, hi)));
}

template <typename T>
void adv_launch(Ctx& c, const LsBatch& b, int scheme, int stage1, double a, double bb, double fdt, const double* vu,
                const double* vv, const double* vw) {
  const T* u = reinterpret_cast<const T*>(vu);
  const T* v = reinterpret_cast<const T*>(vv);
  const T* w = reinterpret_cast<const T*>(vw);
  // one instance per scheme and spacing case (PW: every a/dx a product;
  // the FP32 form always takes the product by the reciprocal)
  const unsigned g = b.start[b.n];
  const bool pw = c.P.pow2 || sizeof(T) == 4;
  if (scheme == ICLS_HOUC5) {
    if (pw) k_adv_stage<ICLS_HOUC5, T, 1><<<g, kTile, 0, c.s>>>(c.P, b, stage1, a, bb, fdt, u, v, w);
    else k_adv_stage<ICLS_HOUC5, T, 0><<<g, kTile, 0, c.s>>>(c.P, b, stage1, a, bb, fdt, u, v, w);
  } else {
    if (pw) k_adv_stage<ICLS_WENO5, T, 1><<<g, kTile, 0, c.s>>>(c.P, b, stage1, a, bb, fdt, u, v, w);
    else k_adv_stage<ICLS_WENO5, T, 0><<<g, kTile, 0, c.s>>>(c.P, b, stage1, a, bb, fdt, u, v, w);
  }
}
// the band list of a batch (its tasks' masks set): entries in c.band_list,
// their number in c.band_count on the device; need = the upper bound the
// caller checked against c.band_cap
void launch_band_list(Ctx& c, const LsBatch& b) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "band_list", 1);
  cudaMemsetAsync(c.band_count, 0, sizeof(int), c.s);
  BandCell* list = reinterpret_cast<BandCell*>(c.band_list);
  BY_FORM(c, (k_band_list<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, list, c.band_count, (int)c.band_cap)),
          (k_band_list<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, list, c.band_count, (int)c.band_cap)));
}
template <typename T>
void adv_split_launch(Ctx& c, const LsBatch& b, int scheme, int stage1, double a, double bb, double fdt,
                      const double* vu, const double* vv, const double* vw, long long need) {
  const T* u = reinterpret_cast<const T*>(vu);
  const T* v = reinterpret_cast<const T*>(vv);
  const T* w = reinterpret_cast<const T*>(vw);
  const BandCell* list = reinterpret_cast<const BandCell*>(c.band_list);
  const unsigned nb = (unsigned)((need + NT - 1) / NT);
  k_adv_base<T><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, stage1, a, bb);
  if (nb > 0) {
    const bool pw = c.P.pow2 || sizeof(T) == 4;
    if (scheme == ICLS_HOUC5) {
      if (pw) k_adv_band<ICLS_HOUC5, T, 1><<<nb, NT, 0, c.s>>>(c.P, b, list, c.band_count, fdt, u, v, w);
      else k_adv_band<ICLS_HOUC5, T, 0><<<nb, NT, 0, c.s>>>(c.P, b, list, c.band_count, fdt, u, v, w);
    } else {
      if (pw) k_adv_band<ICLS_WENO5, T, 1><<<nb, NT, 0, c.s>>>(c.P, b, list, c.band_count, fdt, u, v, w);
      else k_adv_band<ICLS_WENO5, T, 0><<<nb, NT, 0, c.s>>>(c.P, b, list, c.band_count, fdt, u, v, w);
    }
  }
  k_adv_walls<T><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b);
}
// one RK stage over the batch from its band list (launch_band_list first)
void launch_adv_split(Ctx& c, const LsBatch& b, int scheme, int stage1, double a, double bb, double fdt,
                      const double* vu, const double* vv, const double* vw, long long need) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "adv_stage", 3);
  BY_FORM(c, adv_split_launch<float>(c, b, scheme, stage1, a, bb, fdt, vu, vv, vw, need),
          adv_split_launch<double>(c, b, scheme, stage1, a, bb, fdt, vu, vv, vw, need));
}

void launch_adv_stage(Ctx& c, const LsBatch& b, int scheme, int stage1, double a, double bb, double fdt,
                      const double* vu, const double* vv, const double* vw) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "adv_stage", 1);
  BY_FORM(c, adv_launch<float>(c, b, scheme, stage1, a, bb, fdt, vu, vv, vw),
          adv_launch<double>(c, b, scheme, stage1, a, bb, fdt, vu, vv, vw));
}

void launch_reinit_stage(Ctx& c, const LsBatch& b, int stage, double dtau) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "reinit_stage", 1);
  const unsigned g = b.start[b.n];
  // the FP32 form takes the product by the reciprocal at any spacing
  if (c.P.f32) k_reinit_stage<float, 1><<<g, kTile, 0, c.s>>>(c.P, b, stage, dtau, c.drs);
  else if (c.P.pow2) k_reinit_stage<double, 1><<<g, kTile, 0, c.s>>>(c.P, b, stage, dtau, c.drs);
  else k_reinit_stage<double, 0><<<g, kTile, 0, c.s>>>(c.P, b, stage, dtau, c.drs);
}
void launch_reinit_reset(Ctx& c, const LsBatch& b, int maxiter) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "reinit_reset", 1);
  k_reinit_reset<<<1, 64, 0, c.s>>>(b, maxiter, c.drs);
}
void launch_reinit_check(Ctx& c, const LsBatch& b, int it, int maxiter, double thr) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "reinit_check", 1);
  k_reinit_check<<<1, 64, 0, c.s>>>(b, it, maxiter, thr, c.drs, c.dsc, c.P.L - 1);
}

// the per-(tile, chunk) exact sums of H: hcap per drop (4 words each)
XSum* hparts(Ctx& c) { return reinterpret_cast<XSum*>(c.hpart); }

void launch_heaviside(Ctx& c, const LsBatch& b) {
  if (b.n == 0) return;
  Scope sc_(c.prof, c.s, "heaviside", 1);
  BY_FORM(c,
          (k_heaviside<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, reinterpret_cast<float*>(c.jiemian), hparts(c),
                                                                c.hcap)),
          (k_heaviside<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.jiemian, hparts(c), c.hcap)));
}

// n elements of a; tfield: a holds the form's field type (else FP64)
void launch_fill(Ctx& c, double* a, long long n, double v, bool tfield) {
  Scope sc_(c.prof, c.s, "fill", 1);
  if (tfield && c.P.f32)
    k_fill<float><<<1184, NT, 0, c.s>>>(reinterpret_cast<float*>(a), n, v);
  else
    k_fill<double><<<1184, NT, 0, c.s>>>(a, n, v);
}

// outside/ntiles: per drop (null: every drop swept its whole grid)
void launch_disp(Ctx& c, int l) {
  Scope sc_(c.prof, c.s, "disp", 2);
  BY_FORM(c, (k_disp<float><<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, reinterpret_cast<const float*>(c.lv[l]),
                                                                  reinterpret_cast<const float*>(c.ucc),
                                                                  reinterpret_cast<const float*>(c.vcc),
                                                                  reinterpret_cast<const float*>(c.wcc), c.diag)),
          (k_disp<double><<<kRedBlocks, kRedThreads, 0, c.s>>>(c.P, c.lv[l], c.ucc, c.vcc, c.wcc, c.diag)));
  k_disp_final<<<1, kRedThreads, 0, c.s>>>(c.diag, kRedBlocks, c.diag + 7 * kRedBlocks);
}

void launch_materials_final(Ctx& c, const double* outside, const int* ntiles) {
  Scope sc_(c.prof, c.s, "materials_final", 2);
  PerDrop o;
  const int uniform = (outside == nullptr || c.P.L > kMaxDropsParam) ? 1 : 0;
  for (int l = 0; l < kMaxDropsParam; ++l) {
    o.v[l] = (!uniform && l < c.P.L) ? outside[l] : 0.;
    o.n[l] = (!uniform && l < c.P.L) ? ntiles[l] : 0;
  }
  // uniform: every drop swept whole, (kmax + 2) / kStageRows z chunks of
  // red_cap column tiles
  k_volumes<<<1, 1024, 0, c.s>>>(c.P, hparts(c), c.hcap, o, uniform, c.red_cap * ((c.P.kmax + 2) / kHeavRows), c.dvol,
                                c.dsc);
  const int r0[3] = {0, 0, 0}, r1[3] = {c.P.i1, c.P.j1, c.P.k1};
  dim3 g2 = grid_of(r0, r1);
  g2.z = (g2.z + 1) / 2;  // two rows per thread
  if (c.P.f32) {
    auto f = [](double* q) { return reinterpret_cast<float*>(q); };
    if (c.materials_rows1)
      k_materials_final<float><<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, f(c.jiemian), f(c.miu), f(c.rho),
                                                                     f(c.rho_u), f(c.rho_v), f(c.rho_w));
    else
      k_materials_rows2<float><<<g2, kBlock, 0, c.s>>>(c.P, f(c.jiemian), f(c.miu), f(c.rho), f(c.rho_u),
                                                       f(c.rho_v), f(c.rho_w));
  } else {
    if (c.materials_rows1)
      k_materials_final<double><<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, c.jiemian, c.miu, c.rho, c.rho_u,
                                                                      c.rho_v, c.rho_w);
    else
      k_materials_rows2<double><<<g2, kBlock, 0, c.s>>>(c.P, c.jiemian, c.miu, c.rho, c.rho_u, c.rho_v, c.rho_w);
  }
}

// b: one task (shape-C region of the drop, apron 1), phi0 = its level set
void launch_inflate_sums(Ctx& c, const LsBatch& b, double outside) {
  Scope sc_(c.prof, c.s, "inflate_sums", 2);
  double* pa = c.hpart;
  XSum* ph = reinterpret_cast<XSum*>(c.hpart + c.red_cap);
  if (c.P.f32) {
    auto f = [](double* q) { return reinterpret_cast<float*>(q); };
    k_inflate_sums<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, f(c.kappa), f(c.nrm_m), f(c.dheav), pa, ph);
  } else {
    k_inflate_sums<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.kappa, c.nrm_m, c.dheav, pa, ph);
  }
  k_inflate_final<<<1, 32, 0, c.s>>>(c.P, pa, ph, b.start[b.n], b.t[0].l, (double)c.cfg.inflate_step * c.dt, outside,
                                     c.dvol, c.dvol0, c.dmaxchk, c.dsc);
}

// gain-one inflation: phi0 copy, the volume after, and the blend
void launch_region_copy(Ctx& c, const LsBatch& b) {
  Scope sc_(c.prof, c.s, "gain_one", 1);
  BY_FORM(c, (k_region_copy<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b)),
          (k_region_copy<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b)));
}
void launch_gain(Ctx& c, const LsBatch& b, double outside) {
  Scope sc_(c.prof, c.s, "gain_one", 2);
  XSum* ph = reinterpret_cast<XSum*>(c.hpart + c.red_cap);
  BY_FORM(c, (k_region_heav<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, ph)),
          (k_region_heav<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, ph)));
  k_gain_final<<<1, 32, 0, c.s>>>(c.P, ph, b.start[b.n], b.t[0].l, outside, c.dvol, c.dvol0, c.dsc);
}
void launch_volume_now(Ctx& c, const LsBatch& b, double outside) {
  Scope sc_(c.prof, c.s, "gain_one", 2);
  XSum* ph = reinterpret_cast<XSum*>(c.hpart + c.red_cap);
  BY_FORM(c, (k_region_heav<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, ph)),
          (k_region_heav<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, ph)));
  k_volume_now<<<1, 32, 0, c.s>>>(c.P, ph, b.start[b.n], b.t[0].l, outside, c.dvolnow);
}
void launch_region_blend(Ctx& c, const LsBatch& b) {
  Scope sc_(c.prof, c.s, "gain_one", 1);
  BY_FORM(c, (k_region_blend<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.dsc)),
          (k_region_blend<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.dsc)));
}

// b: one task (shape-C region of the drop, apron 0)
void launch_inflate_vel(Ctx& c, const LsBatch& b) {
  Scope sc_(c.prof, c.s, "inflate_vel", 1);
  if (c.P.f32) {
    auto f = [](double* q) { return reinterpret_cast<float*>(q); };
    k_inflate_vel<float><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, f(c.dheav), f(c.kappa), c.dsc, f(c.ulc), f(c.vlc),
                                                           f(c.wlc), c.vin);
  } else {
    k_inflate_vel<double><<<b.start[b.n], kTile, 0, c.s>>>(c.P, b, c.dheav, c.kappa, c.dsc, c.ulc, c.vlc, c.wlc, c.vin);
  }
}

void launch_boundmls(Ctx& c, double* phi) {
  Scope sc_(c.prof, c.s, "boundmls", 1);
  const int r0[3] = {-2, -2, -2}, r1[3] = {c.P.i1 + 2, c.P.j1 + 2, c.P.k1 + 2};
  BY_FORM(c, (k_boundmls<float><<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, reinterpret_cast<float*>(phi))),
          (k_boundmls<double><<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, phi)));
}

void launch_materialize(Ctx& c, const Region& r, double bg, double bgg, double* phi) {
  Scope sc_(c.prof, c.s, "materialize", 1);
  const int r0[3] = {-2, -2, -2}, r1[3] = {c.P.i1 + 2, c.P.j1 + 2, c.P.k1 + 2};
  BY_FORM(c,
          (k_materialize<float><<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, r, bg, bgg, reinterpret_cast<float*>(phi))),
          (k_materialize<double><<<grid_of(r0, r1), kBlock, 0, c.s>>>(c.P, r, bg, bgg, phi)));
}

void launch_copy(Ctx& c, double* dst, const double* src, long long n) {
  Scope sc_(c.prof, c.s, "copy", 1);
  k_copy<double><<<1184, 256, 0, c.s>>>(dst, src, n);
}

void launch_to_float(Ctx& c, double* dst_f32, const double* src, long long n) {
  k_to_float<<<1184, 256, 0, c.s>>>(reinterpret_cast<float*>(dst_f32), src, n);
}
void launch_to_double(Ctx& c, double* dst, const double* src_f32, long long n) {
  k_to_double<<<1184, 256, 0, c.s>>>(dst, reinterpret_cast<const float*>(src_f32), n);
}

}  // namespace icls
