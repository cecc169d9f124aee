// uph_search_neighbors_noalloc: the neighbour search of uph_search_neighbors
// for callers that must not allocate GPU memory -- code that runs inside a
// host application's own memory pool or arena, a real-time loop where an
// allocation could stall, or a plugin host that forbids cudaMalloc after
// start-up.  It works on the caller's device buffers and keeps its scratch
// (the cell histogram, cell starts, cell list and per-query pair counts) in
// one statically sized __device__ array declared below, so a call performs
// no cudaMalloc, cudaFree or other allocation.
//
// Limits: at most kNoAllocMaxParticles particles and kNoAllocMaxCells cells
// of the search grid (cells are as wide as the search radius, over the
// caller's [lo, hi] box), and at most kMaxCellOccupancy particles in one
// cell.  Every GPU that loads the library holds the array (about 12 MiB)
// until the process exits.  All calls share the array, so calls that overlap
// on the GPU (different streams or host threads) race.
//
// Unlike uph_search_neighbors (and the reference's 40-nearest-neighbour
// search), this search is not capped: it returns every in-radius pair.
// Pair offsets and the total are 64-bit, like `cap` and `*niac`.
#include <float.h>
#include <limits.h>
#include <math.h>
#include <string.h>

#include <mutex>
#include <string>

#include "uph_internal.cuh"

namespace uph {

constexpr int kNoAllocMaxParticles = 1 << 18;  // 262,144
constexpr int kNoAllocMaxCells = 1 << 19;      // 524,288
constexpr int kNoAllocScanSums = (kNoAllocMaxCells + 4095) / 4096 + 1;
constexpr int kNoAllocMaxDevices = 64;

// scratch layout, in ints; 64-bit regions start on an even int offset
constexpr size_t even(size_t k) { return (k + 1) & ~size_t(1); }
constexpr size_t kOffCount = 0;                                       // int [ncell]
constexpr size_t kOffStart = kOffCount + kNoAllocMaxCells;            // int [ncell + 1]
constexpr size_t kOffFill = kOffStart + kNoAllocMaxCells + 1;         // int [ncell]
constexpr size_t kOffList = kOffFill + kNoAllocMaxCells;              // int [n]
constexpr size_t kOffCellOf = kOffList + kNoAllocMaxParticles;        // int [n]
constexpr size_t kOffPairCnt = kOffCellOf + kNoAllocMaxParticles;     // int [n_fluid]
constexpr size_t kOffPairOff = even(kOffPairCnt + kNoAllocMaxParticles);          // int64 [n_fluid + 1]
constexpr size_t kOffScan = kOffPairOff + 2 * (kNoAllocMaxParticles + 1);         // int [scan sums]
constexpr size_t kOffScan64 = even(kOffScan + kNoAllocScanSums);                  // int64 [scan sums]
constexpr size_t kOffWords = kOffScan64 + 2 * kNoAllocScanSums;                   // error word, pad
constexpr size_t kScratchInts = kOffWords + 64;

static __device__ __align__(256) int g_noalloc_scratch[kScratchInts];

namespace {

struct NoAllocGrid {
  double lo_x, lo_y, inv_cell, r2cut;
  int ncx, ncy, n_fluid, n_all, pb;
};

__global__ void k_na_keys(NoAllocGrid g, const double *__restrict__ pos, int *__restrict__ cell_of,
                          int *__restrict__ cnt, unsigned *err)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.n_all) return;
  const double fx = (pos[2 * s] - g.lo_x) * g.inv_cell, fy = (pos[2 * s + 1] - g.lo_y) * g.inv_cell;
  int cx = 0, cy = 0;
  if (fx >= 0.0 && fy >= 0.0 && fx < (double)g.ncx && fy < (double)g.ncy) {
    cx = (int)fx;
    cy = (int)fy;
  } else {
    atomicOr(err, ERR_OUT_OF_DOMAIN);
    if (fx > 0.0) cx = (int)fmin(fx, (double)(g.ncx - 1));
    if (fy > 0.0) cy = (int)fmin(fy, (double)(g.ncy - 1));
  }
  const int c = cy * g.ncx + cx;
  cell_of[s] = c;
  atomicAdd(&cnt[c], 1);
}

__global__ void k_na_scatter(NoAllocGrid g, const int *__restrict__ cell_of, const int *__restrict__ start,
                             int *fill, int *__restrict__ list)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.n_all) return;
  const int c = cell_of[s];
  list[start[c] + atomicAdd(&fill[c], 1)] = s;
}

// a cell with more than kMaxCellOccupancy ids is not sorted: it flags a
// neighbour overflow, and the pair kernels then do nothing
__global__ void k_na_sort_cells(const int *__restrict__ start, int *__restrict__ list, int ncell, unsigned *err)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int a = start[c], b = start[c + 1];
  if (b - a > kMaxCellOccupancy) {
    atomicOr(err, ERR_NEIGHBOR_OVERFLOW);
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

__device__ __forceinline__ double na_r2(double dx, double dy) { return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)); }

// The 3 x 3 cells around a query, each cell's ids ascending.
struct NaBlock {
  int k[9], e[9];
};

__device__ __forceinline__ void na_block(const NoAllocGrid &g, const int *__restrict__ start,
                                         const int *__restrict__ list, int c, int s, NaBlock &B)
{
  const int cx = c % g.ncx, cy = c / g.ncx;
#pragma unroll
  for (int q = 0; q < 9; q++) {
    const int xx = cx + q % 3 - 1, yy = cy + q / 3 - 1;
    if (xx < 0 || yy < 0 || xx >= g.ncx || yy >= g.ncy) {
      B.k[q] = B.e[q] = 0;
      continue;
    }
    // first id > s by bisection: ids <= s never form a pair with query s
    int lo = start[yy * g.ncx + xx], hi = start[yy * g.ncx + xx + 1];
    B.e[q] = hi;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (list[mid] <= s)
        lo = mid + 1;
      else
        hi = mid;
    }
    B.k[q] = lo;
  }
}

// pass 0: count each query's pairs; pass 1: write them in ascending j by a
// 9-way merge of the (sorted) cell lists -- O(candidates) per query, with
// no reordering of what is already written.  Counts per query are int
// (at most 9 kMaxCellOccupancy candidates); offsets are 64-bit.
template <bool kWrite>
__global__ void k_na_pairs(NoAllocGrid g, const double *__restrict__ pos, const int *__restrict__ cell_of,
                           const int *__restrict__ start, const int *__restrict__ list, int *__restrict__ cnt,
                           const long long *__restrict__ off, int64_t cap, int32_t *i_pair, int32_t *j_pair,
                           double *rij2, const unsigned *err)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.n_fluid) return;
  if (*err & ERR_NEIGHBOR_OVERFLOW) {  // an overcrowded cell: no walk
    if (!kWrite) cnt[s] = 0;
    return;
  }
  const double xs = pos[2 * s], ys = pos[2 * s + 1];
  NaBlock B;
  na_block(g, start, list, cell_of[s], s, B);
  if (!kWrite) {
    int n = 0;
#pragma unroll
    for (int q = 0; q < 9; q++)
      for (int k = B.k[q]; k < B.e[q]; k++) {
        const int j = list[k];
        if (j >= g.pb) break;  // ids ascend: the rest of the cell is excluded too
        const double r2 = na_r2(xs - pos[2 * j], ys - pos[2 * j + 1]);
        n += (r2 < g.r2cut && r2 > DBL_EPSILON);
      }
    cnt[s] = n;
    return;
  }
  const long long base = off[s];
  long long o = base;
  int head[9];
#pragma unroll
  for (int q = 0; q < 9; q++) head[q] = B.k[q] < B.e[q] ? list[B.k[q]] : INT_MAX;
  for (;;) {
    int j = INT_MAX, qm = 0;
#pragma unroll
    for (int q = 0; q < 9; q++)
      if (head[q] < j) {
        j = head[q];
        qm = q;
      }
    if (j >= g.pb) break;  // every remaining head is excluded (or exhausted)
#pragma unroll
    for (int q = 0; q < 9; q++)
      if (q == qm) {
        B.k[q]++;
        head[q] = B.k[q] < B.e[q] ? list[B.k[q]] : INT_MAX;
      }
    const double r2 = na_r2(xs - pos[2 * j], ys - pos[2 * j + 1]);
    if (!(r2 < g.r2cut && r2 > DBL_EPSILON)) continue;
    if (o >= 0 && o < cap) {
      i_pair[o] = s;
      j_pair[o] = j;
      rij2[o] = r2;
    }
    o++;
  }
}

std::mutex g_setup_mutex;
struct ScratchAddress {
  void *ctx;
  int *ptr;
};
ScratchAddress g_scratch[kNoAllocMaxDevices] = {};

// the calling thread's current driver context (nullptr when it cannot be
// read): a device reset replaces the context and re-registers the module,
// which moves g_noalloc_scratch
void *current_context()
{
  typedef int (*CtxGetCurrent)(void **);
  static CtxGetCurrent fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrent)f;
  });
  void *ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of g_noalloc_scratch for the current device.  Host code
// cannot use the symbol's name as a pointer (on the host it names a
// stand-in, not device memory), so the address is looked up once per device
// (and again if that device's context was replaced), with that device
// current, and reused afterwards.
uph_status scratch_address(int **out)
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(UPH_BAD_ARG, "device ordinal out of range");
  // cudaFree(0) makes the runtime's context current without allocating
  e = cudaFree(nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFree(nullptr)");
  void *ctx = current_context();
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  ScratchAddress &a = g_scratch[dev];
  if (!a.ptr || a.ctx != ctx) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    a.ptr = (int *)p;
    a.ctx = ctx;
  }
  *out = a.ptr;
  return UPH_OK;
}

}  // namespace
}  // namespace uph

using namespace uph;

extern "C" uph_status uph_search_neighbors_noalloc(const double *position, int32_t n_fluid, int32_t n_all,
                                                   int32_t particle_boundary, double dist, const double lo[2],
                                                   const double hi[2], int64_t cap, int32_t *i_pair,
                                                   int32_t *j_pair, double *rij2, int64_t *niac, void *stream)
{
  if (!position || !niac || !lo || !hi || n_fluid < 0 || n_all < n_fluid)
    return fail(UPH_BAD_ARG, "uph_search_neighbors_noalloc: bad arguments");
  *niac = 0;
  if (n_all > kNoAllocMaxParticles)
    return fail(UPH_BAD_ARG, "uph_search_neighbors_noalloc: " + std::to_string(n_all) + " particles exceed the limit of " +
                                 std::to_string(kNoAllocMaxParticles));
  if (!(dist > 0.0) || !(hi[0] > lo[0]) || !(hi[1] > lo[1]))
    return fail(UPH_BAD_ARG, "uph_search_neighbors_noalloc: dist must be positive and hi > lo");
  if (cap > 0 && (!i_pair || !j_pair || !rij2))
    return fail(UPH_BAD_ARG, "uph_search_neighbors_noalloc: output arrays are required when cap > 0");
  NoAllocGrid g;
  const double cell = sqrt(dist) * (1.0 + 1e-9);
  const double nx = ceil((hi[0] - lo[0]) / cell), ny = ceil((hi[1] - lo[1]) / cell);
  if (nx * ny > (double)kNoAllocMaxCells)
    return fail(UPH_BAD_ARG, "uph_search_neighbors_noalloc: the [lo, hi] box needs " + std::to_string((long long)(nx * ny)) +
                                 " cells of the search radius; the limit is " + std::to_string(kNoAllocMaxCells));
  g.lo_x = lo[0];
  g.lo_y = lo[1];
  g.inv_cell = 1.0 / cell;
  g.r2cut = dist;
  g.ncx = (int)fmax(nx, 1.0);
  g.ncy = (int)fmax(ny, 1.0);
  g.n_fluid = n_fluid;
  g.n_all = n_all;
  g.pb = particle_boundary;
  const int ncell = g.ncx * g.ncy;
  int *scratch = nullptr;
  uph_status st = scratch_address(&scratch);
  if (st != UPH_OK) return st;
  if (n_fluid == 0 || n_all == 0) return UPH_OK;
  cudaStream_t q = (cudaStream_t)stream;
  int *count = scratch + kOffCount, *start = scratch + kOffStart, *fill = scratch + kOffFill;
  int *list = scratch + kOffList, *cell_of = scratch + kOffCellOf, *pcnt = scratch + kOffPairCnt;
  long long *poff = reinterpret_cast<long long *>(scratch + kOffPairOff);
  int *sums = scratch + kOffScan;
  long long *sums64 = reinterpret_cast<long long *>(scratch + kOffScan64);
  unsigned *err = (unsigned *)(scratch + kOffWords);
  // the array keeps the previous call's contents: clear what must start at zero
  UPH_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * ncell, q));
  UPH_CUDA(cudaMemsetAsync(fill, 0, sizeof(int) * ncell, q));
  UPH_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), q));
  const int tb = 256;
  k_na_keys<<<(n_all + tb - 1) / tb, tb, 0, q>>>(g, position, cell_of, count, err);
  launch_exclusive_scan(count, start, ncell, sums, q);
  k_na_scatter<<<(n_all + tb - 1) / tb, tb, 0, q>>>(g, cell_of, start, fill, list);
  k_na_sort_cells<<<(ncell + tb - 1) / tb, tb, 0, q>>>(start, list, ncell, err);
  k_na_pairs<false><<<(n_fluid + tb - 1) / tb, tb, 0, q>>>(g, position, cell_of, start, list, pcnt, nullptr, 0,
                                                           nullptr, nullptr, nullptr, err);
  launch_exclusive_scan64(pcnt, poff, n_fluid, sums64, q);
  if (cap > 0)
    k_na_pairs<true><<<(n_fluid + tb - 1) / tb, tb, 0, q>>>(g, position, cell_of, start, list, pcnt, poff, cap,
                                                            i_pair, j_pair, rij2, err);
  UPH_CUDA(cudaGetLastError());
  long long total = 0;
  unsigned errw = 0;
  UPH_CUDA(cudaMemcpyAsync(&total, poff + n_fluid, sizeof(long long), cudaMemcpyDeviceToHost, q));
  UPH_CUDA(cudaMemcpyAsync(&errw, err, sizeof(unsigned), cudaMemcpyDeviceToHost, q));
  UPH_CUDA(cudaStreamSynchronize(q));
  *niac = total;
  if (errw & ERR_OUT_OF_DOMAIN)
    return fail(UPH_OUT_OF_DOMAIN, "uph_search_neighbors_noalloc: a particle lies outside [lo, hi]");
  if (errw & ERR_NEIGHBOR_OVERFLOW) {
    *niac = 0;
    return fail(UPH_NEIGHBOR_OVERFLOW, "uph_search_neighbors_noalloc: a search cell holds more than " +
                                           std::to_string(kMaxCellOccupancy) + " particles");
  }
  if (total > cap)
    return fail(UPH_NEIGHBOR_OVERFLOW, "uph_search_neighbors_noalloc: " + std::to_string(total) +
                                           " pairs do not fit the capacity " + std::to_string(cap));
  return UPH_OK;
}
