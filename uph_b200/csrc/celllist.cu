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
#include <algorithm>


#include "cell_build.cuh"

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

// ---- the build as one cooperative launch ---------------------------------------

__global__ void __launch_bounds__(kCellBuildThreads) k_cell_build(const CellBuildArgs A)
{
  __shared__ int s_off[kCellBuildMaxBlocks + 1];
  __shared__ int s_wt[33];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (A.stats.niac) {
      *A.stats.niac = 0ull;
      *A.stats.max_nb = 0;
    }
    if (A.step_counter) *A.step_counter += 1;
  }
  // the list from the last build is still complete: nothing to do (every
  // block reads the flag before any block can clear it, in phase 4)
  if (A.rebuild && *(volatile unsigned *)A.rebuild == 0u) return;
  cell_build_phases(A, s_off, s_wt);
}

uph_status launch_cell_build(const DevParams &P, const double *x, const double *y, int first, int count,
                             CellGrid &G, unsigned *err, bool storage_order, const PassStats *stats,
                             cudaStream_t s, bool check_rebuild, int *step_counter, const int *dyn_count)
{
  // co-resident blocks: the cooperative launch refuses a grid that does not fit
  static int max_blocks[64] = {};
  int dev = 0;
  UPH_CUDA(cudaGetDevice(&dev));
  int mb = (dev >= 0 && dev < 64) ? max_blocks[dev] : 0;
  if (mb == 0) {
    int sms = 0, per_sm = 0;
    UPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    UPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cell_build, kCellBuildThreads, 0));
    mb = std::min(sms * std::min(per_sm, 2), kCellBuildMaxBlocks);
    if (mb < 1) return fail(UPH_CUDA_ERROR, "the cell-list build kernel cannot be resident");
    if (dev >= 0 && dev < 64) max_blocks[dev] = mb;
  }
  const int want = std::max((count + kCellBuildThreads - 1) / kCellBuildThreads,
                            (G.ncell + 4 * kCellBuildThreads - 1) / (4 * kCellBuildThreads));
  const int blocks = std::max(1, std::min(mb, want));
  CellBuildArgs A;
  A.P = P;
  A.x = x;
  A.y = y;
  A.first = first;
  A.count = std::max(count, 0);
  A.G = G;
  A.err = err;
  A.storage_order = storage_order ? 1 : 0;
  A.rebuild = check_rebuild ? P.rebuild : nullptr;
  A.xbin = P.xbin;
  A.ybin = P.ybin;
  A.stats = stats ? *stats : PassStats{nullptr, nullptr};
  A.step_counter = step_counter;
  A.dyn_count = dyn_count;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kCellBuildThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  UPH_CUDA(cudaLaunchKernelEx(&cfg, k_cell_build, A));
  return UPH_OK;
}


}  // namespace uph
