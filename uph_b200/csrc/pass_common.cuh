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

// Walks the (2 reach + 1)^2 cells around a particle in a fixed order: rows
// bottom to top, cells left to right, each cell's slots in ascending order.
// The cells of one row are consecutive in the cell list, so a row is a single
// range of list positions.
struct NeighbourCursor {
  int cx0, cx1, cy, cy1, ncx, k, kend;
  const int *start;

  __device__ __forceinline__ void init(const DevParams &P, const CellGrid &G, int cell)
  {
    const int cx = cell % P.ncx, cyy = cell / P.ncx;
    cx0 = max(cx - P.reach, 0);
    cx1 = min(cx + P.reach, P.ncx - 1);
    cy = max(cyy - P.reach, 0);
    cy1 = min(cyy + P.reach, P.ncy - 1);
    ncx = P.ncx;
    start = G.start;
    k = start[cy * ncx + cx0];
    kend = start[cy * ncx + cx1 + 1];
  }
  // moves to the next non-empty row range; false when the stencil is exhausted
  __device__ __forceinline__ bool advance()
  {
    while (k >= kend) {
      if (++cy > cy1) return false;
      k = start[cy * ncx + cx0];
      kend = start[cy * ncx + cx1 + 1];
    }
    return true;
  }
  // advances to the next candidate list position; false when exhausted
  __device__ __forceinline__ bool next(int &pos)
  {
    if (!advance()) return false;
    pos = k++;
    return true;
  }
  // up to kBatch candidates of the current range; returns how many, 0 when exhausted
  template <int kBatch>
  __device__ __forceinline__ int next_batch(int &pos)
  {
    if (!advance()) return 0;
    pos = k;
    const int n = min(kBatch, kend - k);
    k += n;
    return n;
  }
};

// Lists the in-radius partners of particle `a` (position xa, ya, reference
// index oa) that form a pair of the reference's list, kNbChunk at a time,
// into column `tid` of `s_nb`.  `on_candidate(b, ob, r2, dx, dy)` sees every
// candidate inside the radius first (for the brute-force wall modes).
// Candidates are tested four at a time so their loads overlap.
template <typename OnCandidate>
__device__ __forceinline__ int list_partners(const DevParams &P, const SlotArrays &S, const CellGrid &G,
                                             NeighbourCursor &cur, bool &more, int a, int oa, double xa, double ya,
                                             unsigned (*s_nb)[kPassThreads], int tid, unsigned &my_pairs,
                                             int &my_nb, OnCandidate on_candidate)
{
  constexpr int kB = 4;
  int cnt = 0;
  while (more && cnt <= kNbChunk - kB) {
    int pos;
    const int n = cur.next_batch<kB>(pos);
    if (n == 0) {
      more = false;
      break;
    }
    int b[kB];
    double bx[kB], by[kB];
#pragma unroll
    for (int u = 0; u < kB; u++) b[u] = (u < n) ? G.list[pos + u] : a;
#pragma unroll
    for (int u = 0; u < kB; u++) {
      bx[u] = S.x[b[u]];
      by[u] = S.y[b[u]];
    }
#pragma unroll
    for (int u = 0; u < kB; u++) {
      if (b[u] == a) continue;
      const double dxa = xa - bx[u], dya = ya - by[u];
      const double r2 = exact_r2(dxa, dya);
      if (!(r2 < P.r2cut)) continue;
      const int ob = S.orig[b[u]];
      on_candidate(b[u], ob, r2, dxa, dya);
      if (r2 <= DBL_EPSILON) continue;
      my_nb++;
      if (max(oa, ob) >= P.pb) continue;
      const bool isI = ob > oa;
      my_pairs += isI;
      s_nb[cnt++][tid] = (unsigned)b[u] | (isI ? kRoleI : 0u);
    }
  }
  return cnt;
}

// LeonnardJonesBoundaryForces (mode 1, derivatives.c:1184-1211) and
// MonaghanBoundaryForce (default mode, :1919-1953): every fluid particle
// against every boundary particle, no pair-list filter.
__device__ __forceinline__ void brute_wall_force(const DevParams &P, double r2, double dxa, double dya, double mb,
                                                 double &fx, double &fy)
{
  if (P.boundary_force == 1) {
    const double r0 = P.dx;
    if (r2 < r0 * r0) {
      double rr = r0 / sqrt(r2);
      rr *= rr;
      rr *= rr;
      const double pb = P.lj_coeff * rr * (rr * rr - 1.) / r2;
      fx += pb * dxa;
      fy += pb * dya;
    }
  } else {
    const double r = sqrt(r2);
    const double q = r / P.h;
    double phi = 0.0;
    if (q >= 0.0 && q < 2.0) {
      const double t = 2.0 - q;
      phi = 0.125 * (1.0 + 1.5 * q) * t * t * t;
    }
    const double gama = P.mach_c * P.mach_c / (P.rho0 * P.dx * P.dy);
    const double c = gama * phi * mb / r2;
    fx += c * dxa;
    fy += c * dya;
  }
}

}  // namespace uph
