// Pieces shared by the rate passes.
#pragma once

#include <float.h>

#include "uph_internal.cuh"

namespace uph {

constexpr int kPassThreads = 128;  // threads per block of a rate pass
constexpr int kNbChunk = 32;       // neighbours listed per thread before they are processed
constexpr unsigned kRoleI = 0x80000000u;  // list-entry flag: this particle is the pair's i

__device__ __forceinline__ double exact_r2(double dx, double dy)
{
  // dx*dx + dy*dy rounded like the reference (no fused multiply-add), so the
  // pair test r2 < (h h) 4 decides exactly as SearchNeighbors does
  return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

// 1/x by Newton-Raphson refinement of the hardware's approximate FP64
// reciprocal (rcp.approx.ftz.f64): two iterations y <- y + y (1 - x y) square
// the relative error each time, from about 2^-23 to below 2^-52.  For the
// normal, finite, non-zero operands of the rate passes this is within one
// ulp of 1/x; it skips the special-case handling of IEEE division.
__device__ __forceinline__ double rcp_nr(double x)
{
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// Walks the 3 x 3 cells around a particle in a fixed order: rows bottom to
// top, cells left to right, each cell's slots in ascending order.
struct NeighbourCursor {
  int cx0, cx1, cy, cy1, ncx, k, kend;
  const int *start;

  __device__ __forceinline__ void init(const DevParams &P, const CellGrid &G, int cell)
  {
    const int cx = cell % P.ncx, cyy = cell / P.ncx;
    cx0 = max(cx - 1, 0);
    cx1 = min(cx + 1, P.ncx - 1);
    cy = max(cyy - 1, 0);
    cy1 = min(cyy + 1, P.ncy - 1);
    ncx = P.ncx;
    start = G.start;
    // one row of adjacent cells is one contiguous range of the cell list
    k = start[cy * ncx + cx0];
    kend = start[cy * ncx + cx1 + 1];
  }
  // advances to the next candidate list position; false when exhausted
  __device__ __forceinline__ bool next(int &pos)
  {
    while (k >= kend) {
      if (++cy > cy1) return false;
      k = start[cy * ncx + cx0];
      kend = start[cy * ncx + cx1 + 1];
    }
    pos = k++;
    return true;
  }
};

}  // namespace uph
