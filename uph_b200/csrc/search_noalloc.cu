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
// caller's [lo, hi] box).  Every GPU that loads the library holds the array
// (about 10 MiB) until the process exits.  All calls share the array, so
// calls that overlap on the GPU (different streams or host threads) race.
#include <float.h>
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

// scratch layout, in ints
constexpr size_t kOffCount = 0;
constexpr size_t kOffStart = kOffCount + kNoAllocMaxCells;          // ncell + 1
constexpr size_t kOffFill = kOffStart + kNoAllocMaxCells + 1;
constexpr size_t kOffList = kOffFill + kNoAllocMaxCells;
constexpr size_t kOffCellOf = kOffList + kNoAllocMaxParticles;
constexpr size_t kOffPairCnt = kOffCellOf + kNoAllocMaxParticles;   // n_fluid + 1
constexpr size_t kOffPairOff = kOffPairCnt + kNoAllocMaxParticles + 1;  // n_fluid + 1
constexpr size_t kOffScan = kOffPairOff + kNoAllocMaxParticles + 1;
constexpr size_t kOffWords = kOffScan + kNoAllocScanSums;            // error word, pad
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

// pass 0: count each query's pairs; pass 1: write them (ascending j, because
// cells are visited in row order and each cell's list is sorted -- the rows
// of the 3 x 3 block are merged below to keep the output sorted by j)
template <bool kWrite>
__global__ void k_na_pairs(NoAllocGrid g, const double *__restrict__ pos, const int *__restrict__ cell_of,
                           const int *__restrict__ start, const int *__restrict__ list, int *__restrict__ cnt,
                           const int *__restrict__ off, int64_t cap, int32_t *i_pair, int32_t *j_pair, double *rij2,
                           const unsigned *err)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.n_fluid) return;
  if (*err & ERR_NEIGHBOR_OVERFLOW) {  // an overcrowded cell: no walk
    if (!kWrite) cnt[s] = 0;
    return;
  }
  const double xs = pos[2 * s], ys = pos[2 * s + 1];
  const int c = cell_of[s], cx = c % g.ncx, cy = c / g.ncx;
  int n = 0;
  const int base = kWrite ? off[s] : 0;
  for (int yy = max(cy - 1, 0); yy <= min(cy + 1, g.ncy - 1); yy++) {
    const int k0 = start[yy * g.ncx + max(cx - 1, 0)], k1 = start[yy * g.ncx + min(cx + 1, g.ncx - 1) + 1];
    for (int k = k0; k < k1; k++) {
      const int j = list[k];
      if (j <= s || j >= g.pb) continue;
      const double r2 = na_r2(xs - pos[2 * j], ys - pos[2 * j + 1]);
      if (!(r2 < g.r2cut && r2 > DBL_EPSILON)) continue;
      if (kWrite) {
        // insertion into the query's segment keeps it sorted by j
        const int64_t o = (int64_t)base + n;
        if (o < cap) {
          int64_t p = o;
          while (p > base && j_pair[p - 1] > j) {
            j_pair[p] = j_pair[p - 1];
            rij2[p] = rij2[p - 1];
            p--;
          }
          i_pair[o] = s;
          j_pair[p] = j;
          rij2[p] = r2;
        }
      }
      n++;
    }
  }
  if (!kWrite) cnt[s] = n;
}

std::mutex g_setup_mutex;
int *g_scratch_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch for the current device.  Host code
// cannot use the symbol's name as a pointer (on the host it names a
// stand-in, not device memory), so the address is looked up once per device
// with that device current and reused afterwards.
uph_status scratch_address(int **out)
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(UPH_BAD_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_ptr[dev] = (int *)p;
  }
  *out = g_scratch_ptr[dev];
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
  int *poff = scratch + kOffPairOff, *sums = scratch + kOffScan;
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
  launch_exclusive_scan(pcnt, poff, n_fluid, sums, q);
  if (cap > 0)
    k_na_pairs<true><<<(n_fluid + tb - 1) / tb, tb, 0, q>>>(g, position, cell_of, start, list, pcnt, poff, cap,
                                                            i_pair, j_pair, rij2, err);
  UPH_CUDA(cudaGetLastError());
  int total = 0;
  unsigned errw = 0;
  UPH_CUDA(cudaMemcpyAsync(&total, poff + n_fluid, sizeof(int), cudaMemcpyDeviceToHost, q));
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
