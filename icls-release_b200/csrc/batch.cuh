// batch.cuh — device helpers of the batched per-drop launches.
//
// A batched launch carries up to kTasks drops (LsTask, ctx.h) in one
// __grid_constant__ kernel parameter.  Its 1-D grid is the concatenation of
// the drops' blocks: block b belongs to the task whose [start, next start)
// holds b, and within the task it is one TBX x TBY column tile times one
// chunk of z rows.  Each thread owns one column of the tile and walks the
// rows of its chunk upwards.
//
// Periodic images: a thread that writes interior column (i,j) also writes
// every halo cell that is a periodic copy of it (three layers in shape L,
// one in shape C), so the halos of every written column stay equal to
// their source columns without a boundary pass.
#pragma once
#include <climits>

#include "ctx.h"

namespace icls {

__device__ __forceinline__ int task_of(const LsBatch& B) {
  const int blk = (int)blockIdx.x;
  int lo = 0, hi = B.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (B.start[mid] <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// the column and the rows of one thread of a batched launch
struct Col {
  int X, Y;    // offsets into the written spans
  int i, j;    // interior column (1..imax, 1..jmax)
  int ka, kb;  // rows of this block's chunk
  int tile;    // column tile index within the task
  int ch;      // z chunk index within the task
  bool ok;     // inside the written spans
  bool cxy;    // a computed column
};
// Flat tasks: block bx of a chunk takes the region's written columns
// 256 bx .. 256 bx + 255 in row-major order (x fastest), so a region of any
// width fills whole warps; otherwise a block is a TBX x TBY column tile.
__device__ __forceinline__ Col col_of(const Params& p, const LsTask& t, int local) {
  Col c;
  const int bx = local % t.tx;
  const int r = local / t.tx;
  const int by = r % t.ty;
  const int ch = r / t.ty;
  c.tile = bx + t.tx * by;
  c.ch = ch;
  if (t.flat) {
    const int col = bx * (TBX * TBY) + (int)threadIdx.x + TBX * (int)threadIdx.y;
    c.Y = col / t.r.xn;
    c.X = col - c.Y * t.r.xn;
  } else {
    c.X = bx * TBX + (int)threadIdx.x;
    c.Y = by * TBY + (int)threadIdx.y;
  }
  c.ok = c.X < t.r.xn && c.Y < t.r.yn;
  c.i = t.r.xa + c.X;
  if (c.i > p.imax) c.i -= p.imax;
  c.j = t.r.ya + c.Y;
  if (c.j > p.jmax) c.j -= p.jmax;
  c.ka = t.r.z0 + ch * t.kc;
  c.kb = (ch == t.nch - 1) ? t.r.z1 : c.ka + t.kc - 1;
  c.cxy = c.X >= t.r.cx0 && c.X <= t.r.cx1 && c.Y >= t.r.cy0 && c.Y <= t.r.cy1;
  return c;
}
__device__ __forceinline__ bool computed(const Col& c, const Region& r, int k) {
  return c.cxy && k >= r.cz0 && k <= r.cz1;
}

// the halo copy of column i in an array with H halo layers, INT_MIN if none
template <int H>
__device__ __forceinline__ int image_of(int i, int n) {
  return i <= H ? i + n : (i > n - H ? i - n : INT_MIN);
}
// v into column (i,j) of row k and its periodic images, shape L
template <typename T>
__device__ __forceinline__ void putL(const Params& p, T* __restrict__ a, int i, int j, int k, T v) {
  const int ii = image_of<3>(i, p.imax), jj = image_of<3>(j, p.jmax);
  a[idxL(p, i, j, k)] = v;
  if (ii != INT_MIN) a[idxL(p, ii, j, k)] = v;
  if (jj != INT_MIN) {
    a[idxL(p, i, jj, k)] = v;
    if (ii != INT_MIN) a[idxL(p, ii, jj, k)] = v;
  }
}
// the same for shape C (one halo layer)
template <typename T>
__device__ __forceinline__ void putC(const Params& p, T* __restrict__ a, int i, int j, int k, T v) {
  const int ii = image_of<1>(i, p.imax), jj = image_of<1>(j, p.jmax);
  a[idxC(p, i, j, k)] = v;
  if (ii != INT_MIN) a[idxC(p, ii, j, k)] = v;
  if (jj != INT_MIN) {
    a[idxC(p, i, jj, k)] = v;
    if (ii != INT_MIN) a[idxC(p, ii, jj, k)] = v;
  }
}
// storage cell (i,j,k) of shape L (halo coordinates allowed) is written by r
__device__ __forceinline__ bool in_written(const Params& p, const Region& r, int i, int j, int k) {
  return k >= r.z0 && k <= r.z1 && span_has(r.xa, r.xn, p.imax, wrapx(p, i)) &&
         span_has(r.ya, r.yn, p.jmax, wrapy(p, j));
}

// the field type T view of a task's type-erased level-set pointers
template <typename T>
__device__ __forceinline__ const T* cT(const double* q) { return reinterpret_cast<const T*>(q); }
template <typename T>
__device__ __forceinline__ T* mT(double* q) { return reinterpret_cast<T*>(q); }

}  // namespace icls
