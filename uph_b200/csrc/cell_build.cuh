// The phases of the one-launch cell-list build (celllist.cu).
#pragma once

#include "uph_internal.cuh"

namespace uph {

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *warp_tot, T &total)
{
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    T wv = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : T(0);
    T wi = wv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warp_tot[lane] = wi - wv;  // exclusive prefix of warp totals
    if (lane == 31) warp_tot[32] = wi;
  }
  __syncthreads();
  const T out = incl - v + warp_tot[wid];
  total = warp_tot[32];
  __syncthreads();
  return out;
}


struct CellBuildArgs {
  DevParams P;
  const double *x, *y;
  int first, count;
  CellGrid G;
  unsigned *err;
  int storage_order;
  unsigned *rebuild;  // non-null: skip unless set; clear it and record the binned positions
  double *xbin, *ybin;
  PassStats stats;    // non-null niac: zeroed for the rate pass that follows, built or not
  int *step_counter;  // non-null: advanced by one, built or not
  const int *dyn_count;  // non-null: the ids are [first, first + min(count, *dyn_count))
};

// Grid-wide barrier over co-resident blocks: arrive on bar[0]; the last
// block resets it and bumps the generation bar[1]; the others wait for the
// bump.  The wait gives up after kWaitNs on the global timer (setting
// ERR_TIMEOUT); the result is uniform over the block.
__device__ __forceinline__ bool cell_grid_barrier(unsigned *bar, unsigned *err)
{
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned *vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicAdd(&bar[1], 1u);
    } else {
      const unsigned long long t0 = global_ns();
      long long polls = 0;
      while (*vgen == gen) {
        if ((++polls & 255) == 0 && global_ns() - t0 > kWaitNs) {
          atomicOr(err, ERR_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ int cell_of_position(const DevParams &P, double px, double py, unsigned *err,
                                                bool storage_order)
{
  const double fx = (px - P.lo_x) * P.inv_cell;
  const double fy = (py - P.lo_y) * P.inv_cell;
  const bool inside = px >= P.lo_x && py >= P.lo_y && px <= P.hi_x && py <= P.hi_y;
  int cx = 0, cy = 0;
  if (inside) {
    cx = min((int)floor(fx), P.ncx - 1);
    cy = min((int)floor(fy), P.ncy - 1);
  } else {
    atomicOr(err, ERR_OUT_OF_DOMAIN);
    if (fx > 0.0) cx = (int)fmin(fx, (double)(P.ncx - 1));
    if (fy > 0.0) cy = (int)fmin(fy, (double)(P.ncy - 1));
  }
  return storage_order ? storage_key(cx, cy, P.ntx, P.tile) : cy * P.ncx + cx;
}

// Phases (B = grid barrier):
//   1. cell of every slot, histogram; a slot's rank in its cell is the
//      value its atomic add returned                                    B
//   2. each block scans its chunk of cells: local prefixes into fill[],
//      the chunk's total into totals[]; count is zeroed as it is read     B
//   3. every block scans totals[] in shared memory, writes the final
//      start[] of its chunk and scatters its slots to
//      fill[c] + offset(chunk of c) + rank                               B
//   4. each cell's slots sorted ascending (insertion sort, short cells),
//      so the order does not depend on atomic arrival order; a cell with
//      more than kMaxCellOccupancy slots is left unsorted and flags a
//      neighbour overflow.
// The same formulas as the multi-launch build (k_cell_keys and the rest).
// The build's phases for any block size; s_off: shared memory for
// gridDim.x + 1 ints, s_wt: 33 ints.  False when a grid barrier gave up.
// Every block of the (co-resident) grid must call it.
__device__ __forceinline__ bool cell_build_phases(const CellBuildArgs &A, int *s_off, int *s_wt)
{
  const int nb = gridDim.x, b = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
  const int stride = nb * nt;
  const int count = A.dyn_count ? min(A.count, *A.dyn_count) : A.count;
  const int ncell = A.G.ncell;
  int *cnt = A.G.count, *start = A.G.start, *fill = A.G.fill, *list = A.G.list;
  int *cell_of = A.G.cell_of, *rank = A.G.rank;

  // 1. keys and histogram
  for (int k = b * nt + t; k < count; k += stride) {
    const int s = A.first + k;
    const double px = A.x[s], py = A.y[s];
    const int c = cell_of_position(A.P, px, py, A.err, A.storage_order != 0);
    cell_of[s] = c;
    rank[s] = atomicAdd(&cnt[c], 1);
    if (A.rebuild) {
      A.xbin[s] = px;
      A.ybin[s] = py;
    }
  }
  if (!cell_grid_barrier(A.G.bar, A.err)) return false;

  // 2. chunk scans
  const int chunk = (ncell + nb - 1) / nb;
  const int c0 = min(b * chunk, ncell), c1 = min(c0 + chunk, ncell);
  int carry = 0;
  for (int base = c0; base < c1; base += nt * 4) {
    int v[4], sum = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = base + t * 4 + j;
      v[j] = 0;
      if (c < c1) {
        v[j] = cnt[c];
        cnt[c] = 0;
      }
      sum += v[j];
    }
    int total;
    int run = block_exclusive_scan<int>(sum, s_wt, total) + carry;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = base + t * 4 + j;
      if (c < c1) fill[c] = run;
      run += v[j];
    }
    carry += total;
  }
  if (t == 0) A.G.totals[b] = carry;
  if (!cell_grid_barrier(A.G.bar, A.err)) return false;

  // 3. chunk offsets, final starts, scatter
  {
    int run = 0;
    for (int base = 0; base < nb; base += nt) {
      const int i = base + t;
      const int v = i < nb ? A.G.totals[i] : 0;
      int total;
      const int ex = block_exclusive_scan<int>(v, s_wt, total);
      if (i < nb) s_off[i] = ex + run;
      run += total;
    }
    if (t == 0) s_off[nb] = run;
    __syncthreads();
  }
  for (int c = c0 + t; c < c1; c += nt) start[c] = fill[c] + s_off[b];
  if (b == nb - 1 && t == 0) start[ncell] = s_off[nb];
  for (int k = b * nt + t; k < count; k += stride) {
    const int s = A.first + k;
    const int c = cell_of[s];
    list[fill[c] + s_off[c / chunk] + rank[s]] = s;
  }
  if (!cell_grid_barrier(A.G.bar, A.err)) return false;

  // 4. per-cell sort by slot
  if (b == 0 && t == 0) {
    if (A.rebuild) *A.rebuild = 0u;
    if (A.G.gen) *A.G.gen += 1u;  // the passes' candidate lists are stale
  }
  for (int c = b * nt + t; c < ncell; c += stride) {
    const int a0 = start[c], a1 = start[c + 1];
    if (a1 - a0 > kMaxCellOccupancy) {
      atomicOr(A.err, ERR_NEIGHBOR_OVERFLOW);
      continue;
    }
    for (int i = a0 + 1; i < a1; i++) {
      const int v = list[i];
      int j = i - 1;
      while (j >= a0 && list[j] > v) {
        list[j + 1] = list[j];
        j--;
      }
      list[j + 1] = v;
    }
  }
  return true;
}

}  // namespace uph
