// Cell list: the GPU replacement of the reference's kd-tree search
// (src/lib/Search.cc:5-44).  Every step the interacting particles are binned
// into square cells of radius / reach by a counting sort:
//   1. cell key per slot + histogram (atomic add per cell),
//   2. exclusive scan of the histogram -> first entry of every cell,
//   3. scatter of slot ids into their cell's range,
//   4. sort of every cell's (short) range by slot id, so the order in which
//      the pair pass visits neighbours -- and with it every floating-point
//      sum -- does not depend on atomic arrival order.
// A particle's neighbours then lie within `reach` cells of its own (a
// (2 reach + 1)^2 block; reach 2, cells of half the radius, by default).
#include "uph_internal.cuh"

namespace uph {

// storage_order = false: row-major cell ids for the cell list;
// storage_order = true: tile-major keys for sorting the particle storage.
__global__ void k_cell_keys(DevParams P, const double *__restrict__ x, const double *__restrict__ y, int first,
                            int count, int *__restrict__ cell_of, int *__restrict__ cnt, unsigned *err,
                            bool storage_order)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int s = first + k;
  const double px = x[s], py = y[s];
  const double fx = (px - P.lo_x) * P.inv_cell;
  const double fy = (py - P.lo_y) * P.inv_cell;
  // the declared domain [lo, hi]; NaN positions fail the comparisons too
  const bool inside = px >= P.lo_x && py >= P.lo_y && px <= P.hi_x && py <= P.hi_y;
  int cx = 0, cy = 0;
  if (inside) {
    cx = min((int)floor(fx), P.ncx - 1);
    cy = min((int)floor(fy), P.ncy - 1);
  } else {
    atomicOr(err, ERR_OUT_OF_DOMAIN);
    // clamp into the grid so the cell list stays well formed
    if (fx > 0.0) cx = (int)fmin(fx, (double)(P.ncx - 1));
    if (fy > 0.0) cy = (int)fmin(fy, (double)(P.ncy - 1));
  }
  const int c = storage_order ? storage_key(cx, cy, P.ntx, P.tile) : cy * P.ncx + cx;
  cell_of[s] = c;
  atomicAdd(&cnt[c], 1);
}

void launch_cell_keys(const DevParams &P, const double *x, const double *y, int first, int count, CellGrid &G,
                      unsigned *err, bool storage_order, cudaStream_t s)
{
  if (count <= 0) return;
  k_cell_keys<<<(count + 255) / 256, 256, 0, s>>>(P, x, y, first, count, G.cell_of, G.count, err, storage_order);
}

// ---- exclusive scan ----------------------------------------------------------
// Three passes over chunks of SCAN_CHUNK ints: chunk sums, a scan of the
// chunk sums in one block, then the chunk-local scans plus their offsets.
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER_THREAD = 4;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_PER_THREAD;

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

// In: counts of type C; out, the chunk sums and the running totals: type T
// (int for cell histograms, long long for pair counts that may pass 2^31).
template <typename C, typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_chunk_sums(const C *__restrict__ in, int n,
                                                                  T *__restrict__ sums)
{
  __shared__ T wt[33];
  const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER_THREAD;
  T v = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++)
    if (base + k < n) v += (T)in[base + k];
  T total;
  block_exclusive_scan<T>(v, wt, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(T *sums, int nsums)
{
  __shared__ T wt[33];
  T carry = 0;
  for (int base = 0; base < nsums; base += SCAN_THREADS) {
    const int i = base + threadIdx.x;
    const T v = (i < nsums) ? sums[i] : T(0);
    T total;
    const T ex = block_exclusive_scan<T>(v, wt, total);
    if (i < nsums) sums[i] = ex + carry;
    carry += total;
  }
}

template <typename C, typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_chunks(const C *__restrict__ in, T *__restrict__ out,
                                                              int n, const T *__restrict__ sums)
{
  __shared__ T wt[33];
  const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER_THREAD;
  T v[SCAN_PER_THREAD];
  T tsum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++) {
    v[k] = (base + k < n) ? (T)in[base + k] : T(0);
    tsum += v[k];
  }
  T total;
  T run = block_exclusive_scan<T>(tsum, wt, total) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  // out[n] = grand total, written by the thread that owns element n-1
  if (base <= n - 1 && n - 1 < base + SCAN_PER_THREAD) out[n] = run;
}

int scan_block_sums_needed(int n) { return (n + SCAN_CHUNK - 1) / SCAN_CHUNK; }

void launch_exclusive_scan(const int *in, int *out, int n, int *block_sums, cudaStream_t s)
{
  const int nb = scan_block_sums_needed(n);
  k_scan_chunk_sums<int, int><<<nb, SCAN_THREADS, 0, s>>>(in, n, block_sums);
  k_scan_sums<int><<<1, SCAN_THREADS, 0, s>>>(block_sums, nb);
  k_scan_chunks<int, int><<<nb, SCAN_THREADS, 0, s>>>(in, out, n, block_sums);
}

void launch_exclusive_scan64(const int *in, long long *out, int n, long long *block_sums, cudaStream_t s)
{
  const int nb = scan_block_sums_needed(n);
  k_scan_chunk_sums<int, long long><<<nb, SCAN_THREADS, 0, s>>>(in, n, block_sums);
  k_scan_sums<long long><<<1, SCAN_THREADS, 0, s>>>(block_sums, nb);
  k_scan_chunks<int, long long><<<nb, SCAN_THREADS, 0, s>>>(in, out, n, block_sums);
}

__global__ void k_cell_scatter(const int *__restrict__ cell_of, const int *__restrict__ start, int *fill,
                               int *__restrict__ list, int first, int count)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int s = first + k;
  const int c = cell_of[s];
  list[start[c] + atomicAdd(&fill[c], 1)] = s;
}

void launch_cell_scatter(const CellGrid &G, int first, int count, cudaStream_t s)
{
  if (count <= 0) return;
  k_cell_scatter<<<(count + 255) / 256, 256, 0, s>>>(G.cell_of, G.start, G.fill, G.list, first, count);
}

// Each cell's ids ascending (insertion sort by one thread).  A cell holding
// more than kMaxCellOccupancy ids is not sorted: it flags a neighbour
// overflow instead, which bounds this kernel's work on pathological inputs
// (a radius of the whole domain, particles piled into a border cell).
__global__ void k_cell_sort_segments(const int *__restrict__ start, int *__restrict__ list, int ncell, unsigned *err)
{
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int a = start[c], b = start[c + 1];
  if (b - a > kMaxCellOccupancy) {
    if (err) atomicOr(err, ERR_NEIGHBOR_OVERFLOW);
    return;
  }
  for (int i = a + 1; i < b; i++) {
    const int v = list[i];
    int j = i - 1;
    while (j >= a && list[j] > v) {
      list[j + 1] = list[j];
      j--;
    }
    list[j + 1] = v;
  }
}

void launch_cell_sort_segments(const CellGrid &G, unsigned *err, cudaStream_t s)
{
  k_cell_sort_segments<<<(G.ncell + 255) / 256, 256, 0, s>>>(G.start, G.list, G.ncell, err);
}

}  // namespace uph
