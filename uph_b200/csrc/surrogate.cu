// Learned surrogate (include/uph_surrogate.h): the message-passing network's
// forward and backward passes, Adam, and the judged coupling to a simulation.
//
// Data layout in HBM, nodes row-major (one row per node, padded to 128
// columns where a tensor-core K granule needs it):
//   graph   nbr[n][32] int32 partners (cell-list order), ef[n][32] float4
//           ((dx, dy, r)/R, (rho_j - rho_i)/(rho0 s_e))
//   F[n][128] BF16 features, a1[n][128] BF16
//   per round: cat[n][256] BF16 = [h | m] (h, the residual stream, is BF16:
//              each residual add is FP32, then rounded), PQ[n][256] BF16, S[n][128] BF16,
//              u[n][128] BF16
//   out[n][128] FP32 (5 columns used)
// Node-local layers are BF16 GEMMs on the tcgen05 tensor cores: for training
// one GEMM per layer with every activation stored (tc_gemm.cu); for
// inference fused per round, a tile of nodes going through all of a round's
// layers on chip (node_chain.cu).
// The edge layer is a warp per receiving node: lane l owns channels
// [4l, 4l + 4); partner indices and edge features are loaded by lane k for
// partner k and broadcast by shuffles; Q_j rows are 256-byte coalesced
// gathers (the slot order is spatially sorted, so they mostly hit L2).
// Sums over partners run in the graph's (deterministic) partner order and all reductions
// (bias and W_e gradients, loss) use fixed grids and fixed orders, so a
// forward/backward pass is bitwise reproducible.
#include <cuda_bf16.h>
#include <float.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "node_chain.cuh"
#include "sim_access.cuh"
#include "uph_internal.cuh"
#include "uph_surrogate.h"

namespace uph {
namespace {

constexpr int kLat = UPH_SUR_LATENT;
constexpr int kFeat = 128;
constexpr int kOutPad = 128;
constexpr int kNOut = UPH_SUR_OUTPUTS;
constexpr int kMaxDeg = UPH_SUR_MAX_DEGREE;
constexpr int kMaxRounds = UPH_SUR_MAX_ROUNDS;
constexpr int kEdgeThreads = 256;           // 8 warps
// fixed grid (per-warp partials in a fixed order) of one wave: the edge
// kernels take 80 registers x 256 threads, so three blocks fit an SM's 64K
// registers; a fourth block per SM would run as a second, mostly empty wave
constexpr int kEdgeBlocks = 148 * 3;
constexpr int kColBlocks = 148 * 2;         // bias-gradient partial sums
constexpr int kSplitMax = 148;              // split-K CTAs of one weight-gradient GEMM tile
constexpr int kLossBlocks = 148;
constexpr int kMaxBins = 4096;

typedef __nv_bfloat16 bf16;

// ---- parameter layout --------------------------------------------------------
struct RoundOff {
  size_t pq_w, pq_b, we, w2, n1_w, n1_b, n2_w, n2_b;
};
struct ParamOff {
  size_t enc1_w, enc1_b, enc2_w, enc2_b;
  RoundOff r[kMaxRounds];
  size_t dec1_w, dec1_b, dec2_w, dec2_b;
  size_t total;
};

ParamOff param_layout(int rounds)
{
  ParamOff o{};
  size_t p = 0;
  auto take = [&](size_t n) {
    size_t at = p;
    p += n;
    return at;
  };
  o.enc1_w = take(kLat * kFeat);
  o.enc1_b = take(kLat);
  o.enc2_w = take(kLat * kLat);
  o.enc2_b = take(kLat);
  for (int r = 0; r < rounds; r++) {
    o.r[r].pq_w = take(2 * kLat * kLat);
    o.r[r].pq_b = take(2 * kLat);
    o.r[r].we = take(kLat * 4);
    o.r[r].w2 = take(kLat * kLat);
    o.r[r].n1_w = take(kLat * 2 * kLat);
    o.r[r].n1_b = take(kLat);
    o.r[r].n2_w = take(kLat * kLat);
    o.r[r].n2_b = take(kLat);
  }
  o.dec1_w = take(kLat * kLat);
  o.dec1_b = take(kLat);
  o.dec2_w = take(kOutPad * kLat);
  o.dec2_b = take(kOutPad);
  o.total = p;
  return o;
}

// ---- small device helpers ------------------------------------------------------
__device__ __forceinline__ void load_bf16x4(const bf16 *p, float out[4])
{
  const uint2 raw = *reinterpret_cast<const uint2 *>(p);
  const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(&raw.x);
  const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162 *>(&raw.y);
  const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
  out[0] = fa.x;
  out[1] = fa.y;
  out[2] = fb.x;
  out[3] = fb.y;
}

__device__ __forceinline__ void store_bf16x4(bf16 *p, const float v[4])
{
  __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]);
  __nv_bfloat162 b = __floats2bfloat162_rn(v[2], v[3]);
  uint2 raw;
  raw.x = *reinterpret_cast<uint32_t *>(&a);
  raw.y = *reinterpret_cast<uint32_t *>(&b);
  *reinterpret_cast<uint2 *>(p) = raw;
}

// the edge pre-activation, one fixed operation order shared by the forward
// and backward kernels so both see bit-identical values
__device__ __forceinline__ float edge_z(float p, float q, const float4 &w, float e0, float e1, float e2, float e3)
{
  return __fmaf_rn(w.w, e3, __fmaf_rn(w.z, e2, __fmaf_rn(w.y, e1, __fmaf_rn(w.x, e0, __fadd_rn(p, q)))));
}

// packed FP32 pairs (sm_100 f32x2 instructions): each half rounds exactly
// like the scalar FP32 operation, so packed and scalar code agree bitwise
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pack2(float lo, float hi)
{
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}

__device__ __forceinline__ void unpack2(f32x2 v, float &lo, float &hi)
{
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c)
{
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b)
{
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// two BF16 values (one 32-bit word) as an FP32 pair
__device__ __forceinline__ f32x2 bf2_to_f2(uint32_t w)
{
  return pack2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}

__device__ __forceinline__ f32x2 relu2(f32x2 v)
{
  float a, b;
  unpack2(v, a, b);
  return pack2(fmaxf(a, 0.0f), fmaxf(b, 0.0f));
}

// ---- graph --------------------------------------------------------------------
// partners of every node within R (DBL_EPSILON < r^2 < R^2) in cell-list
// order (cells row by row, ids ascending inside a cell: deterministic), and
// their edge features in FP32: (dx, dy, r) / R and the density difference
// (rho_j - rho_i) / rho_unit
__global__ void k_sur_graph(DevParams G, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ rho, double rho_unit, int n, const int *__restrict__ cell_of,
                            const int *__restrict__ start, const int *__restrict__ list, double R,
                            int *__restrict__ nbr, float4 *__restrict__ ef, int *__restrict__ deg, unsigned *err)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[i], yi = y[i], ri = rho[i];
  const double r2cut = R * R;
  // features by multiplication with reciprocals (no FP64 division or square
  // root per edge); they are rounded to FP32 anyway
  const double inv_R = 1.0 / R, inv_R2 = 1.0 / r2cut, inv_rho_unit = 1.0 / rho_unit;
  const int c = cell_of[i];
  const int cx = c % G.ncx, cy = c / G.ncx;
  int cnt = 0;
  for (int oy = -1; oy <= 1; oy++) {
    const int yy = cy + oy;
    if (yy < 0 || yy >= G.ncy) continue;
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, G.ncx - 1);
    const int a = start[yy * G.ncx + x0], b = start[yy * G.ncx + x1 + 1];
    // four candidates per pass: their position loads are independent
    for (int k0 = a; k0 < b; k0 += 4) {
      int jj[4];
      double cx4[4], cy4[4];
#pragma unroll
      for (int u = 0; u < 4; u++) jj[u] = k0 + u < b ? list[k0 + u] : -1;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        cx4[u] = jj[u] >= 0 ? x[jj[u]] : 0.0;
        cy4[u] = jj[u] >= 0 ? y[jj[u]] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int j = jj[u];
        if (j < 0) continue;
        const double dx = cx4[u] - xi, dy = cy4[u] - yi;
        const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        if (r2 > DBL_EPSILON && r2 < r2cut) {
          if (cnt < kMaxDeg) {
            nbr[(size_t)i * kMaxDeg + cnt] = j;
            ef[(size_t)i * kMaxDeg + cnt] = make_float4((float)(dx * inv_R), (float)(dy * inv_R),
                                                        sqrtf((float)(r2 * inv_R2)),
                                                        (float)((rho[j] - ri) * inv_rho_unit));
          }
          cnt++;
        }
      }
    }
  }
  if (cnt > kMaxDeg) {
    atomicOr(err, ERR_NEIGHBOR_OVERFLOW);
    cnt = kMaxDeg;
  }
  deg[i] = cnt;
}

// ---- features -----------------------------------------------------------------
__global__ void k_sur_features(int n, const double *__restrict__ u, const double *__restrict__ v,
                               const double *__restrict__ rho, const int32_t *__restrict__ itype, double vel_scale,
                               double rho0, double rho_scale, bf16 *__restrict__ F, unsigned *err)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = itype[i];
  float f[8];
  f[0] = (float)(u[i] / vel_scale);
  f[1] = (float)(v[i] / vel_scale);
  f[2] = (float)((rho[i] / rho0 - 1.0) / rho_scale);
  f[3] = t == 1 ? 1.0f : 0.0f;
  f[4] = (t != 1 && t != 3) ? 1.0f : 0.0f;
  f[5] = t == 3 ? 1.0f : 0.0f;
  f[6] = 0.0f;
  f[7] = 0.0f;
  if (!isfinite(f[0]) || !isfinite(f[1]) || !isfinite(f[2])) atomicOr(err, ERR_NAN);
  __align__(16) __nv_bfloat162 h[4];
  for (int k = 0; k < 4; k++) h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
  uint4 *row = reinterpret_cast<uint4 *>(F + (size_t)i * kFeat);
  row[0] = *reinterpret_cast<uint4 *>(&h[0]);
  for (int k = 1; k < kFeat / 8; k++) row[k] = make_uint4(0u, 0u, 0u, 0u);
}

// ---- edge layer -----------------------------------------------------------------
// S_i = sum_j relu(P_i + Q_j + W_e e_ij), PQ rows = [P | Q].  A half-warp
// per node, lane l of the half owning channels [8l, 8l + 8) as four packed
// FP32 pairs (the operation order of edge_z).  Each warp stages its two
// nodes' edge records (features + partner) in shared memory, so a partner
// costs one shared broadcast read and one 16-byte gather of its Q row;
// partners are summed in graph order.
__global__ void __launch_bounds__(kEdgeThreads) k_sur_edge_fwd(int n, const bf16 *__restrict__ PQ,
                                                                 const float *__restrict__ we,
                                                                 const int *__restrict__ nbr,
                                                                 const float4 *__restrict__ ef,
                                                                 const int *__restrict__ deg, bf16 *__restrict__ S)
{
  __shared__ float4 rec[kEdgeThreads / 32][2][kMaxDeg];
  __shared__ int recj[kEdgeThreads / 32][2][kMaxDeg];
  const int lane = threadIdx.x & 31, hl = lane & 15, half = lane >> 4, wib = threadIdx.x >> 5;
  const int gh = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;  // global half-warp
  const int nh = (gridDim.x * blockDim.x) >> 4;
  const int c0 = hl * 8;
  f32x2 w0[4], w1[4], w2[4], w3[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const float4 wa = *reinterpret_cast<const float4 *>(we + (c0 + 2 * q) * 4);
    const float4 wb = *reinterpret_cast<const float4 *>(we + (c0 + 2 * q + 1) * 4);
    w0[q] = pack2(wa.x, wb.x);
    w1[q] = pack2(wa.y, wb.y);
    w2[q] = pack2(wa.z, wb.z);
    w3[q] = pack2(wa.w, wb.w);
  }
  float4 *my = rec[wib][half];
  int *myj = recj[wib][half];
  const int passes = (n + nh - 1) / nh;  // the same for both halves of a warp
  for (int ps = 0; ps < passes; ps++) {
    const int i = gh + ps * nh;
    const bool live = i < n;
    const int d = live ? deg[i] : 0;
    __syncwarp();  // the last pass's records are read
    for (int k = hl; k < d; k += 16) {
      my[k] = ef[(size_t)i * kMaxDeg + k];
      myj[k] = nbr[(size_t)i * kMaxDeg + k];
    }
    __syncwarp();
    f32x2 p[4], acc[4];
    {
      uint4 praw = make_uint4(0u, 0u, 0u, 0u);
      if (live) praw = *reinterpret_cast<const uint4 *>(PQ + (size_t)i * 2 * kLat + c0);
      p[0] = bf2_to_f2(praw.x);
      p[1] = bf2_to_f2(praw.y);
      p[2] = bf2_to_f2(praw.z);
      p[3] = bf2_to_f2(praw.w);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) acc[q] = pack2(0.0f, 0.0f);
    int k = 0;
    for (; k + 4 <= d; k += 4) {
      float4 e[4];
      uint4 qv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) e[u] = my[k + u];
#pragma unroll
      for (int u = 0; u < 4; u++)
        qv[u] = *reinterpret_cast<const uint4 *>(PQ + (size_t)myj[k + u] * 2 * kLat + kLat + c0);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const f32x2 e0 = pack2(e[u].x, e[u].x), e1 = pack2(e[u].y, e[u].y), e2 = pack2(e[u].z, e[u].z);
        const f32x2 e3 = pack2(e[u].w, e[u].w);
        const uint32_t qw[4] = {qv[u].x, qv[u].y, qv[u].z, qv[u].w};
#pragma unroll
        for (int q = 0; q < 4; q++)
          acc[q] = add2(acc[q], relu2(fma2(w3[q], e3, fma2(w2[q], e2, fma2(w1[q], e1,
                                                                              fma2(w0[q], e0, add2(p[q], bf2_to_f2(qw[q]))))))));
      }
    }
    for (; k < d; k++) {
      const float4 e = my[k];
      const uint4 qv = *reinterpret_cast<const uint4 *>(PQ + (size_t)myj[k] * 2 * kLat + kLat + c0);
      const f32x2 e0 = pack2(e.x, e.x), e1 = pack2(e.y, e.y), e2 = pack2(e.z, e.z), e3 = pack2(e.w, e.w);
      const uint32_t qw[4] = {qv.x, qv.y, qv.z, qv.w};
#pragma unroll
      for (int q = 0; q < 4; q++)
        acc[q] = add2(acc[q], relu2(fma2(w3[q], e3, fma2(w2[q], e2, fma2(w1[q], e1,
                                                                            fma2(w0[q], e0, add2(p[q], bf2_to_f2(qw[q]))))))));
    }
    if (live) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 4; q++) unpack2(acc[q], v[2 * q], v[2 * q + 1]);
      __align__(16) __nv_bfloat162 h[4];
#pragma unroll
      for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
      *reinterpret_cast<uint4 *>(S + (size_t)i * kLat + c0) = *reinterpret_cast<uint4 *>(&h[0]);
    }
  }
}

// gradients of the edge layer, node a as receiver (dP_a, dW_e) and as sender
// (dQ_a, through every partner b that receives from a: the graph is
// symmetric and e_ba = (-e_ab.x, -e_ab.y, e_ab.z))
__global__ void __launch_bounds__(kEdgeThreads) k_sur_edge_bwd(int n, const bf16 *__restrict__ PQ,
                                                                 const float *__restrict__ we,
                                                                 const int *__restrict__ nbr,
                                                                 const float4 *__restrict__ ef,
                                                                 const int *__restrict__ deg,
                                                                 const float *__restrict__ dS, bf16 *__restrict__ dPQ,
                                                                 float *__restrict__ we_part)
{
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int c0 = lane * 4;
  float4 w[4];
  for (int c = 0; c < 4; c++) w[c] = *reinterpret_cast<const float4 *>(we + (c0 + c) * 4);
  float g[4][4];
  for (int c = 0; c < 4; c++) g[c][0] = g[c][1] = g[c][2] = g[c][3] = 0.0f;
  for (int a = gw; a < n; a += nw) {
    const int d = deg[a];
    int myj = 0;
    float4 mye = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane < d) {
      myj = nbr[(size_t)a * kMaxDeg + lane];
      mye = ef[(size_t)a * kMaxDeg + lane];
    }
    float pa[4], qa[4];
    load_bf16x4(PQ + (size_t)a * 2 * kLat + c0, pa);
    load_bf16x4(PQ + (size_t)a * 2 * kLat + kLat + c0, qa);
    const float4 dsa4 = *reinterpret_cast<const float4 *>(dS + (size_t)a * kLat + c0);
    const float dsa[4] = {dsa4.x, dsa4.y, dsa4.z, dsa4.w};
    float dp[4] = {0.f, 0.f, 0.f, 0.f}, dq[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < d; k++) {
      const int b = __shfl_sync(0xffffffffu, myj, k);
      const float e0 = __shfl_sync(0xffffffffu, mye.x, k);
      const float e1 = __shfl_sync(0xffffffffu, mye.y, k);
      const float e2 = __shfl_sync(0xffffffffu, mye.z, k);
      const float e3 = __shfl_sync(0xffffffffu, mye.w, k);
      float pb[4], qb[4];
      load_bf16x4(PQ + (size_t)b * 2 * kLat + c0, pb);
      load_bf16x4(PQ + (size_t)b * 2 * kLat + kLat + c0, qb);
      const float4 dsb4 = *reinterpret_cast<const float4 *>(dS + (size_t)b * kLat + c0);
      const float dsb[4] = {dsb4.x, dsb4.y, dsb4.z, dsb4.w};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        if (edge_z(pa[c], qb[c], w[c], e0, e1, e2, e3) > 0.0f) {
          dp[c] += dsa[c];
          g[c][0] = __fmaf_rn(dsa[c], e0, g[c][0]);
          g[c][1] = __fmaf_rn(dsa[c], e1, g[c][1]);
          g[c][2] = __fmaf_rn(dsa[c], e2, g[c][2]);
          g[c][3] = __fmaf_rn(dsa[c], e3, g[c][3]);
        }
        // the reverse edge: dx, dy and the density difference change sign
        if (edge_z(pb[c], qa[c], w[c], -e0, -e1, e2, -e3) > 0.0f) dq[c] += dsb[c];
      }
    }
    store_bf16x4(dPQ + (size_t)a * 2 * kLat + c0, dp);
    store_bf16x4(dPQ + (size_t)a * 2 * kLat + kLat + c0, dq);
  }
  // the block's 8 warps summed in warp order: one partial row per block
  __shared__ float4 red[kEdgeThreads / 32][kLat];
  const int wib = threadIdx.x >> 5;
  for (int c = 0; c < 4; c++) red[wib][c0 + c] = make_float4(g[c][0], g[c][1], g[c][2], g[c][3]);
  __syncthreads();
  if (threadIdx.x < kLat) {
    float4 t = red[0][threadIdx.x];
    for (int w = 1; w < kEdgeThreads / 32; w++) {
      const float4 o = red[w][threadIdx.x];
      t.x += o.x;
      t.y += o.y;
      t.z += o.z;
      t.w += o.w;
    }
    reinterpret_cast<float4 *>(we_part)[(size_t)blockIdx.x * kLat + threadIdx.x] = t;
  }
}

// out[c] = sum over rows of part[r][c] in a fixed order: block = 32 columns
// x 32 row lanes, lane l sums rows l, l + 32, ... and the lanes are added in
// lane order (deterministic; 32-way parallel instead of one long chain)
__global__ void __launch_bounds__(1024) k_sum_rows(const float *__restrict__ part, int rows, int cols,
                                                    float *__restrict__ out)
{
  __shared__ float red[32][33];
  const int cl = threadIdx.x & 31, l = threadIdx.x >> 5;
  const int c = blockIdx.x * 32 + cl;
  float s = 0.0f;
  if (c < cols)
    for (int r = l; r < rows; r += 32) s += part[(size_t)r * cols + c];
  red[l][cl] = s;
  __syncthreads();
  if (l == 0 && c < cols) {
    float t = red[0][cl];
    for (int k = 1; k < 32; k++) t += red[k][cl];
    out[c] = t;
  }
}
inline void sum_rows(const float *part, int rows, int cols, float *out, cudaStream_t s)
{
  k_sum_rows<<<(cols + 31) / 32, 1024, 0, s>>>(part, rows, cols, out);
}

// column sums of a BF16 [n x cols] block (ld >= cols): per-block partials
__global__ void k_colsum_part(const bf16 *__restrict__ src, int ld, int cols, int n, int rows_per_block,
                              float *__restrict__ part)
{
  const int c = threadIdx.x;
  if (c >= cols) return;
  const int r0 = blockIdx.x * rows_per_block, r1 = min(n, r0 + rows_per_block);
  float s = 0.0f;
  for (int r = r0; r < r1; r++) s += __bfloat162float(src[(size_t)r * ld + c]);
  part[(size_t)blockIdx.x * cols + c] = s;
}

// mean squared error over the fluid rows' 5 outputs; dO = dL/dout in BF16
// (zero outside the fluid rows and the 5 columns)
__global__ void k_sur_loss(int n, int nf, const float *__restrict__ out, const float *__restrict__ target,
                           float inv_count, bf16 *__restrict__ dO, float *__restrict__ part)
{
  __shared__ float red[256];
  float s = 0.0f;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    float gr[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (r < nf) {
      for (int c = 0; c < kNOut; c++) {
        const float d = out[(size_t)r * kOutPad + c] - target[(size_t)r * kNOut + c];
        s += d * d;
        gr[c] = 2.0f * d * inv_count;
      }
    }
    __align__(16) __nv_bfloat162 h[4];
    for (int k = 0; k < 4; k++) h[k] = __floats2bfloat162_rn(gr[2 * k], gr[2 * k + 1]);
    uint4 *row = reinterpret_cast<uint4 *>(dO + (size_t)r * kOutPad);
    row[0] = *reinterpret_cast<uint4 *>(&h[0]);
    for (int k = 1; k < kOutPad / 8; k++) row[k] = make_uint4(0u, 0u, 0u, 0u);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0] * inv_count;
}

__global__ void k_f32_to_bf16(const float *__restrict__ src, bf16 *__restrict__ dst, size_t count)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) dst[i] = __float2bfloat16_rn(src[i]);
}

__global__ void k_copy_out(int n, const float *__restrict__ out, float *__restrict__ dst)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kNOut) return;
  dst[i] = out[(size_t)(i / kNOut) * kOutPad + i % kNOut];
}

// sum of squared gradients, per-block partials
__global__ void k_sumsq_part(const float *__restrict__ g, size_t count, float *__restrict__ part)
{
  __shared__ float red[256];
  float s = 0.0f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    s += g[i] * g[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adam (bias-corrected), optional global-norm clipping from *sumsq; writes
// the FP32 master weights and their BF16 copy
__global__ void k_adam(size_t count, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, bf16 *__restrict__ wb, float lr, float b1, float b2, float eps,
                       float c1, float c2, const float *__restrict__ sumsq, float clip)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float scale = 1.0f;
  if (clip > 0.0f) {
    const float norm = sqrtf(*sumsq);
    if (norm > clip) scale = clip / norm;
  }
  const float gi = g[i] * scale;
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
}

__device__ __forceinline__ double tait_p(const DevParams &P, double rho)
{
  return P.B * (pow(rho / P.rho0, P.gamma) - 1.0);
}

struct OutScale {
  double T;         // macro_steps * dt
  double s[kNOut];
  double max_move;  // the sanity guard's largest displacement (the graph radius)
  double min_gap;   // smallest fluid-wall distance a prediction may reach (0.25 R)
};

// Threshold of the sanity guard: a prediction whose density leaves
// rho0 (1 +- kMaxRhoDev) is rejected (weakly compressible flow stays within
// about 1 % of rho0).
constexpr double kMaxRhoDev = 0.05;

// network prediction of the fluid slots into pred[orig][5] =
// (x, y, u, v, rho), with the non-penetration projection against the wall
// particles of the current graph; flags *bad when a value is non-finite,
// the density leaves the guard band, or a particle would move more than the
// graph radius or leave the simulation's domain
__global__ void k_sur_predict(DevParams P, SlotArrays S, const float *__restrict__ out, OutScale sc,
                              const int *__restrict__ nbr, const int *__restrict__ deg, double *__restrict__ pred,
                              unsigned *bad)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const float *o = out + (size_t)a * kOutPad;
  const double u = S.u[a], v = S.v[a];
  double x = S.x[a] + sc.T * u + sc.s[0] * o[0];
  double y = S.y[a] + sc.T * v + sc.s[1] * o[1];
  double un = u + sc.s[2] * o[2];
  double vn = v + sc.s[3] * o[3];
  const double rho = S.rho[a] + sc.s[4] * o[4];
  // non-penetration: a predicted position closer than min_gap to a wall
  // particle (advanced by its own velocity) is moved back out to min_gap
  // along the line from that particle, and the velocity loses its component
  // into the wall -- unless the particle already was that close
  const double g2 = sc.min_gap * sc.min_gap;
  for (int k = 0; k < deg[a]; k++) {
    const int j = nbr[(size_t)a * kMaxDeg + k];
    if (S.itype[j] == 1) continue;
    const double wx = S.x[j] + sc.T * S.u[j], wy = S.y[j] + sc.T * S.v[j];
    const double rx = x - wx, ry = y - wy;
    const double dn = rx * rx + ry * ry;
    const double d0 = (S.x[a] - S.x[j]) * (S.x[a] - S.x[j]) + (S.y[a] - S.y[j]) * (S.y[a] - S.y[j]);
    if (dn < g2 && dn < d0 && dn > 0.0) {
      const double d = sqrt(dn), nx = rx / d, ny = ry / d;
      x = wx + nx * sc.min_gap;
      y = wy + ny * sc.min_gap;
      const double vin = (un - S.u[j]) * nx + (vn - S.v[j]) * ny;
      if (vin < 0.0) {
        un -= vin * nx;
        vn -= vin * ny;
      }
    }
  }
  const bool inside = x >= P.lo_x && x <= P.hi_x && y >= P.lo_y && y <= P.hi_y;
  const bool small_move = fabs(x - S.x[a]) <= sc.max_move && fabs(y - S.y[a]) <= sc.max_move;
  if (!isfinite(x) || !isfinite(y) || !isfinite(un) || !isfinite(vn) || !(fabs(rho / P.rho0 - 1.0) <= kMaxRhoDev) ||
      !inside || !small_move)
    atomicOr(bad, 1u);
  double *q = pred + (size_t)S.orig[a] * kNOut;
  q[0] = x;
  q[1] = y;
  q[2] = un;
  q[3] = vn;
  q[4] = rho;
}

// an accepted prediction becomes the fluid state (slots found through their
// reference index, so it survives re-sorts in between); WCSPH pressure is
// the Tait law of the density, the local* fields equal the state
__global__ void k_sur_commit(DevParams P, SlotArrays S, const double *__restrict__ pred)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double *q = pred + (size_t)S.orig[a] * kNOut;
  const double rho = q[4];
  const double p = tait_p(P, rho);
  S.x[a] = q[0];
  S.y[a] = q[1];
  S.u[a] = q[2];
  S.v[a] = q[3];
  S.ut[a] = q[2];
  S.vt[a] = q[3];
  S.rho[a] = rho;
  S.rhot[a] = rho;
  S.p[a] = p;
  S.pt[a] = p;
  S.pressure[a] = p;
}

__device__ __forceinline__ unsigned ordered_bits(float f)
{
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// the judge: density error of the network's prediction against the plain
// solver's state (per particle, matched by reference index) and the highest
// fluid particle of both in every x-bin
__global__ void k_sur_judge(DevParams P, SlotArrays S, const double *__restrict__ pred, double x0, double inv_bin,
                            int nbins, unsigned *__restrict__ bins_plain, unsigned *__restrict__ bins_pred,
                            double *__restrict__ part)
{
  __shared__ double red_s[256], red_m[256];
  double sq = 0.0, mx = 0.0;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P.nf; a += gridDim.x * blockDim.x) {
    const double *q = pred + (size_t)S.orig[a] * kNOut;
    const double rp = S.rho[a];
    const double rel = (q[4] - rp) / rp;
    sq += rel * rel;
    mx = fmax(mx, fabs(rel));
    const double bp = floor((S.x[a] - x0) * inv_bin), bq = floor((q[0] - x0) * inv_bin);
    if (bp >= 0.0 && bp < nbins) atomicMax(&bins_plain[(int)bp], ordered_bits((float)S.y[a]));
    if (bq >= 0.0 && bq < nbins) atomicMax(&bins_pred[(int)bq], ordered_bits((float)q[1]));
  }
  red_s[threadIdx.x] = sq;
  red_m[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      red_s[threadIdx.x] += red_s[threadIdx.x + o];
      red_m[threadIdx.x] = fmax(red_m[threadIdx.x], red_m[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = red_s[0];
    part[2 * blockIdx.x + 1] = red_m[0];
  }
}
constexpr int kJudgeBlocks = 296;

struct NodesView {
  int n, nf;
  const double *x, *y, *u, *v, *rho;
  const int32_t *itype;
  double lo_x, lo_y, hi_x, hi_y;
};

}  // namespace
}  // namespace uph

using namespace uph;

struct uph_surrogate {
  uph_sur_config cfg;
  ParamOff off;
  int cap = 0;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  unsigned *d_err = nullptr;
  unsigned *d_bad = nullptr;  // sanity guard of the last prediction
  // parameters: FP32 master, BF16 copy, gradient, Adam moments
  float *w = nullptr, *g = nullptr, *am = nullptr, *av = nullptr;
  bf16 *wb = nullptr;
  int adam_t = 0;
  // graph
  CellGrid grid{};
  long long grid_cap = 0;
  int *nbr = nullptr, *deg = nullptr;
  float4 *ef = nullptr;
  // activations
  bf16 *F = nullptr, *a1 = nullptr, *d1 = nullptr;
  float *out = nullptr;
  bf16 *cat[kMaxRounds + 1] = {}, *PQ[kMaxRounds] = {}, *S[kMaxRounds] = {}, *u[kMaxRounds] = {};
  // backward
  bf16 *dO = nullptr, *dz = nullptr, *dhb = nullptr, *dm = nullptr, *dPQ = nullptr;
  float *dh = nullptr, *dS = nullptr;
  float *partials = nullptr, *colpart = nullptr, *wepart = nullptr, *losspart = nullptr, *lossval = nullptr;
  float *sqpart = nullptr, *sumsq = nullptr;
  // fused inference path (node_chain.cu): pre-swizzled weight images, the
  // residual stream ping-pong, TMA tensor maps over F, S[0] and h
  uint8_t *wimg = nullptr;
  bool img_dirty = true;
  bool fused = true;
  bf16 *hb[2] = {};
  CUtensorMap tm_F, tm_S, tm_H[2], tm_PQ;
  // judge
  double *pred = nullptr, *jpart = nullptr;
  unsigned *bins = nullptr;
  int n_pred = 0;
  int n_last = 0, nf_last = 0;
  bool have_grad = false;
  // judged coupling: macro steps since the last check, plain macro steps left
  int since_judge = 0;
  int fallback_left = 0;
  int64_t last_sim = 0;  // serial of the simulation the schedule belongs to
};

namespace {

template <typename T>
cudaError_t salloc(uph_surrogate *s, T **p, size_t count)
{
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
  if (e == cudaSuccess) s->allocs.push_back((void *)*p);
  return e;
}

void free_all(uph_surrogate *s)
{
  for (void *p : s->allocs) cudaFree(p);
  s->allocs.clear();
}

uph_status ensure_grid(uph_surrogate *s, long long ncell)
{
  if (ncell <= s->grid_cap) return UPH_OK;
  // only the cell-sized arrays grow; list and cell_of are node-sized (create)
  for (void *p : {(void *)s->grid.count, (void *)s->grid.start, (void *)s->grid.fill, (void *)s->grid.block_sums})
    if (p) cudaFree(p);
  s->grid.count = s->grid.start = s->grid.fill = s->grid.block_sums = nullptr;
  s->grid_cap = 0;
  const long long cap = ncell + ncell / 4 + 1024;
  if (cap > (1LL << 30)) return fail(UPH_BAD_ARG, "surrogate: node box too large for the graph grid");
  UPH_CUDA(cudaMalloc((void **)&s->grid.count, sizeof(int) * cap));
  UPH_CUDA(cudaMalloc((void **)&s->grid.start, sizeof(int) * (cap + 1)));
  UPH_CUDA(cudaMalloc((void **)&s->grid.fill, sizeof(int) * cap));
  const int nb = scan_block_sums_needed((int)cap + 1);
  UPH_CUDA(cudaMalloc((void **)&s->grid.block_sums, sizeof(int) * (nb + 1)));
  s->grid.nblock_sums = nb;
  s->grid_cap = cap;
  return UPH_OK;
}

uph_status check_err(uph_surrogate *s)
{
  unsigned err = 0;
  UPH_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof err, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  UPH_CUDA(cudaGetLastError());
  if (err & ERR_NEIGHBOR_OVERFLOW)
    return fail(UPH_NEIGHBOR_OVERFLOW, "surrogate: a node has more than 32 graph partners");
  if (err & ERR_NAN) return fail(UPH_NAN, "surrogate: a non-finite value in the node state or prediction");
  if (err & ERR_OUT_OF_DOMAIN) return fail(UPH_OUT_OF_DOMAIN, "surrogate: a node lies outside the given box");
  if (err & ERR_TIMEOUT) return fail(UPH_TIMEOUT, "surrogate: a tensor-core wait timed out");
  return UPH_OK;
}

// graph + features for `nv`
uph_status prepare(uph_surrogate *s, const NodesView &nv)
{
  if (nv.n <= 0 || nv.n > s->cap || nv.nf < 0 || nv.nf > nv.n)
    return fail(UPH_BAD_ARG, "surrogate: node count outside [1, capacity]");
  if (!(nv.hi_x > nv.lo_x) || !(nv.hi_y > nv.lo_y)) return fail(UPH_BAD_ARG, "surrogate: empty node box");
  cudaStream_t q = s->stream;
  const double R = s->cfg.radius;
  DevParams G{};
  G.lo_x = nv.lo_x;
  G.lo_y = nv.lo_y;
  G.hi_x = nv.hi_x;
  G.hi_y = nv.hi_y;
  G.cell = R;
  G.inv_cell = 1.0 / R;
  G.ncx = (int)ceil((nv.hi_x - nv.lo_x) / R) + 1;
  G.ncy = (int)ceil((nv.hi_y - nv.lo_y) / R) + 1;
  G.tile = 1;
  G.ntx = G.ncx;
  const long long ncell = (long long)G.ncx * G.ncy;
  uph_status r = ensure_grid(s, ncell);
  if (r != UPH_OK) return r;
  CellGrid &g = s->grid;
  g.ncell = (int)ncell;
  UPH_CUDA(cudaMemsetAsync(g.count, 0, sizeof(int) * ncell, q));
  UPH_CUDA(cudaMemsetAsync(g.fill, 0, sizeof(int) * ncell, q));
  launch_cell_keys(G, nv.x, nv.y, 0, nv.n, g, s->d_err, false, q);
  launch_exclusive_scan(g.count, g.start, (int)ncell, g.block_sums, q);
  launch_cell_scatter(g, 0, nv.n, q);
  launch_cell_sort_segments(g, s->d_err, q);
  k_sur_graph<<<(nv.n + 127) / 128, 128, 0, q>>>(G, nv.x, nv.y, nv.rho, s->cfg.rho0 * s->cfg.edge_rho_scale, nv.n,
                                                 g.cell_of, g.start, g.list, R, s->nbr, s->ef, s->deg, s->d_err);
  k_sur_features<<<(nv.n + 255) / 256, 256, 0, q>>>(nv.n, nv.u, nv.v, nv.rho, nv.itype, s->cfg.vel_scale,
                                                     s->cfg.rho0, s->cfg.rho_scale, s->F, s->d_err);
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

struct Gemm {
  GemmCall c;
  Gemm(const void *A, int lda, const void *B, int ldb, int M, int N, int K)
  {
    c.A = A;
    c.lda = lda;
    c.B = B;
    c.ldb = ldb;
    c.M = M;
    c.N = N;
    c.K = K;
  }
};

uph_status run(uph_surrogate *s, GemmCall c)
{
  c.err = s->d_err;
  return launch_tc_gemm(c, s->stream);
}

// weight gradient dW[M x N] = sum over nodes of dY[node][M-index] X[node][N-index]
uph_status wgrad(uph_surrogate *s, const bf16 *dY, int ldy, int M, const bf16 *X, int ldx, int N, int n, float *dst)
{
  GemmCall c;
  c.A = dY;
  c.lda = ldy;
  c.a_trans = 1;
  c.B = X;
  c.ldb = ldx;
  c.b_trans = 1;
  c.M = M;
  c.N = N;
  c.K = (n + 63) / 64 * 64;
  c.k_valid = n;
  const int tiles = (M / 128) * (N / 128);
  c.splits = std::max(1, std::min(kSplitMax / tiles, c.K / 64));
  c.partials = s->partials;
  c.c_f32 = dst;
  c.ldc = N;
  return run(s, c);
}

uph_status colsum(uph_surrogate *s, const bf16 *src, int ld, int cols, int n, float *dst)
{
  const int rpb = (n + kColBlocks - 1) / kColBlocks;
  k_colsum_part<<<kColBlocks, cols, 0, s->stream>>>(src, ld, cols, n, rpb, s->colpart);
  sum_rows(s->colpart, kColBlocks, cols, dst, s->stream);
  return UPH_OK;
}

#define TRYS(x)                     \
  do {                              \
    uph_status r_ = (x);            \
    if (r_ != UPH_OK) return r_;    \
  } while (0)

uph_status forward_net(uph_surrogate *s, int n)
{
  const ParamOff &o = s->off;
  const float *W = s->w;
  const bf16 *Wb = s->wb;
  cudaStream_t q = s->stream;
  {
    GemmCall c;
    c.A = s->F; c.lda = kFeat; c.B = Wb + o.enc1_w; c.ldb = kFeat;
    c.M = n; c.N = kLat; c.K = kFeat;
    c.bias = W + o.enc1_b; c.relu = 1; c.c_bf16 = s->a1; c.ldc = kLat;
    TRYS(run(s, c));
  }
  {
    GemmCall c;
    c.A = s->a1; c.lda = kLat; c.B = Wb + o.enc2_w; c.ldb = kLat;
    c.M = n; c.N = kLat; c.K = kLat;
    c.bias = W + o.enc2_b; c.c_bf16 = s->cat[0]; c.ldc = 2 * kLat;
    TRYS(run(s, c));
  }
  const int rounds = s->cfg.rounds;
  for (int r = 0; r < rounds; r++) {
    const RoundOff &ro = o.r[r];
    {
      GemmCall c;
      c.A = s->cat[r]; c.lda = 2 * kLat; c.B = Wb + ro.pq_w; c.ldb = kLat;
      c.M = n; c.N = 2 * kLat; c.K = kLat;
      c.bias = W + ro.pq_b; c.c_bf16 = s->PQ[r]; c.ldc = 2 * kLat;
      TRYS(run(s, c));
    }
    k_sur_edge_fwd<<<kEdgeBlocks, kEdgeThreads, 0, q>>>(n, s->PQ[r], W + ro.we, s->nbr, s->ef, s->deg, s->S[r]);
    {
      GemmCall c;
      c.A = s->S[r]; c.lda = kLat; c.B = Wb + ro.w2; c.ldb = kLat;
      c.M = n; c.N = kLat; c.K = kLat;
      c.c_bf16 = s->cat[r] + kLat; c.ldc = 2 * kLat;
      TRYS(run(s, c));
    }
    {
      GemmCall c;
      c.A = s->cat[r]; c.lda = 2 * kLat; c.B = Wb + ro.n1_w; c.ldb = 2 * kLat;
      c.M = n; c.N = kLat; c.K = 2 * kLat;
      c.bias = W + ro.n1_b; c.relu = 1; c.c_bf16 = s->u[r]; c.ldc = kLat;
      TRYS(run(s, c));
    }
    {
      GemmCall c;
      c.A = s->u[r]; c.lda = kLat; c.B = Wb + ro.n2_w; c.ldb = kLat;
      c.M = n; c.N = kLat; c.K = kLat;
      c.bias = W + ro.n2_b; c.residual = s->cat[r]; c.ldr = 2 * kLat;
      c.c_bf16 = s->cat[r + 1]; c.ldc = 2 * kLat;
      TRYS(run(s, c));
    }
  }
  {
    GemmCall c;
    c.A = s->cat[rounds]; c.lda = 2 * kLat; c.B = Wb + o.dec1_w; c.ldb = kLat;
    c.M = n; c.N = kLat; c.K = kLat;
    c.bias = W + o.dec1_b; c.relu = 1; c.c_bf16 = s->d1; c.ldc = kLat;
    TRYS(run(s, c));
  }
  {
    GemmCall c;
    c.A = s->d1; c.lda = kLat; c.B = Wb + o.dec2_w; c.ldb = kLat;
    c.M = n; c.N = kOutPad; c.K = kLat;
    c.bias = W + o.dec2_b; c.c_f32 = s->out; c.ldc = kOutPad;
    TRYS(run(s, c));
  }
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

// the shared-memory images of every weight matrix the fused kernels stream
void build_images(uph_surrogate *s)
{
  const ParamOff &o = s->off;
  auto img = [&](size_t off, int N, int K) { launch_swizzle_image(s->wb + off, N, K, s->wimg + off * sizeof(bf16), s->stream); };
  img(o.enc1_w, kLat, kFeat);
  img(o.enc2_w, kLat, kLat);
  for (int r = 0; r < s->cfg.rounds; r++) {
    // W_pq as two 128 x 128 pieces: the P rows, then the Q rows
    img(o.r[r].pq_w, kLat, kLat);
    img(o.r[r].pq_w + kLat * kLat, kLat, kLat);
    img(o.r[r].w2, kLat, kLat);
    img(o.r[r].n1_w, kLat, 2 * kLat);
    img(o.r[r].n2_w, kLat, kLat);
  }
  img(o.dec1_w, kLat, kLat);
  img(o.dec2_w, kOutPad, kLat);
  s->img_dirty = false;
}

// the same network as forward_net through the fused node-chain kernels:
// one kernel for the encoder and one per round, with the edge layer
// between them; outputs land in s->out (columns 0..15)
uph_status forward_fused(uph_surrogate *s, int n)
{
  const ParamOff &o = s->off;
  const float *W = s->w;
  if (s->img_dirty) build_images(s);
  constexpr size_t kHalf = (size_t)kLat * kLat * sizeof(bf16);  // one 128 x 128 piece image
  auto piece = [&](size_t w_off, size_t byte_off, const float *bias) {
    ChainPiece c;
    c.img = s->wimg + w_off * sizeof(bf16) + byte_off;
    c.bias = bias;
    return c;
  };
  ChainArgs a;
  memset(&a, 0, sizeof a);
  a.n = n;
  a.ntiles = (n + 127) / 128;
  a.err = s->d_err;
  a.mode = CHAIN_ENCODER;
  a.tm_a = s->tm_F;
  a.piece[0] = piece(o.enc1_w, 0, W + o.enc1_b);
  a.piece[1] = piece(o.enc2_w, 0, W + o.enc2_b);
  a.piece[2] = piece(o.r[0].pq_w, 0, nullptr);
  a.piece[3] = piece(o.r[0].pq_w, kHalf, W + o.r[0].pq_b);
  a.tm_hout = s->tm_H[0];
  a.tm_pq = s->tm_PQ;
  a.store_h = 1;
  TRYS(launch_node_chain(a, s->stream));
  const int rounds = s->cfg.rounds;
  for (int r = 0; r < rounds; r++) {
    const RoundOff &ro = o.r[r];
    k_sur_edge_fwd<<<kEdgeBlocks, kEdgeThreads, 0, s->stream>>>(n, s->PQ[0], W + ro.we, s->nbr, s->ef, s->deg,
                                                                s->S[0]);
    const bool last = r == rounds - 1;
    a.mode = last ? CHAIN_LAST : CHAIN_ROUND;
    a.tm_a = s->tm_S;
    a.tm_h = s->tm_H[r & 1];
    a.piece[0] = piece(ro.w2, 0, nullptr);
    a.piece[1] = piece(ro.n1_w, 0, nullptr);
    a.piece[2] = piece(ro.n1_w, kHalf, W + ro.n1_b);
    a.piece[3] = piece(ro.n2_w, 0, W + ro.n2_b);
    if (last) {
      a.piece[4] = piece(o.dec1_w, 0, W + o.dec1_b);
      a.piece[5] = piece(o.dec2_w, 0, W + o.dec2_b);
      a.store_h = 0;
      a.out = s->out;
    } else {
      a.piece[4] = piece(o.r[r + 1].pq_w, 0, nullptr);
      a.piece[5] = piece(o.r[r + 1].pq_w, kHalf, W + o.r[r + 1].pq_b);
      a.tm_hout = s->tm_H[(r + 1) & 1];
      a.store_h = 1;
    }
    TRYS(launch_node_chain(a, s->stream));
  }
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

uph_status forward_any(uph_surrogate *s, int n) { return s->fused ? forward_fused(s, n) : forward_net(s, n); }

// backward from dO (already in s->dO) to s->g
uph_status backward_net(uph_surrogate *s, int n)
{
  const ParamOff &o = s->off;
  const bf16 *Wb = s->wb;
  float *G = s->g;
  cudaStream_t q = s->stream;
  const int rounds = s->cfg.rounds;
  UPH_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * o.total, q));
  // decoder
  TRYS(wgrad(s, s->dO, kOutPad, kOutPad, s->d1, kLat, kLat, n, G + o.dec2_w));
  TRYS(colsum(s, s->dO, kOutPad, kOutPad, n, G + o.dec2_b));
  {
    GemmCall c;  // dz = (dO . Dec2) masked by d1 > 0
    c.A = s->dO; c.lda = kOutPad; c.B = Wb + o.dec2_w; c.ldb = kLat; c.b_trans = 1;
    c.M = n; c.N = kLat; c.K = kOutPad;
    c.mask = s->d1; c.ldm = kLat; c.c_bf16 = s->dz; c.ldc = kLat;
    TRYS(run(s, c));
  }
  TRYS(wgrad(s, s->dz, kLat, kLat, s->cat[rounds], 2 * kLat, kLat, n, G + o.dec1_w));
  TRYS(colsum(s, s->dz, kLat, kLat, n, G + o.dec1_b));
  {
    GemmCall c;  // dh = dz . Dec1
    c.A = s->dz; c.lda = kLat; c.B = Wb + o.dec1_w; c.ldb = kLat; c.b_trans = 1;
    c.M = n; c.N = kLat; c.K = kLat;
    c.c_f32 = s->dh; c.ldc = kLat;
    TRYS(run(s, c));
  }
  const size_t nl = (size_t)n * kLat;
  for (int r = rounds - 1; r >= 0; r--) {
    const RoundOff &ro = o.r[r];
    k_f32_to_bf16<<<(unsigned)((nl + 255) / 256), 256, 0, q>>>(s->dh, s->dhb, nl);
    TRYS(wgrad(s, s->dhb, kLat, kLat, s->u[r], kLat, kLat, n, G + ro.n2_w));
    TRYS(colsum(s, s->dhb, kLat, kLat, n, G + ro.n2_b));
    {
      GemmCall c;  // dz = (dh . N2) masked by u > 0
      c.A = s->dhb; c.lda = kLat; c.B = Wb + ro.n2_w; c.ldb = kLat; c.b_trans = 1;
      c.M = n; c.N = kLat; c.K = kLat;
      c.mask = s->u[r]; c.ldm = kLat; c.c_bf16 = s->dz; c.ldc = kLat;
      TRYS(run(s, c));
    }
    TRYS(wgrad(s, s->dz, kLat, kLat, s->cat[r], 2 * kLat, 2 * kLat, n, G + ro.n1_w));
    TRYS(colsum(s, s->dz, kLat, kLat, n, G + ro.n1_b));
    {
      GemmCall c;  // dh += dz . N1[:, :128]
      c.A = s->dz; c.lda = kLat; c.B = Wb + ro.n1_w; c.ldb = 2 * kLat; c.b_trans = 1;
      c.M = n; c.N = kLat; c.K = kLat;
      c.accumulate = 1; c.c_f32 = s->dh; c.ldc = kLat;
      TRYS(run(s, c));
    }
    {
      GemmCall c;  // dm = dz . N1[:, 128:]
      c.A = s->dz; c.lda = kLat; c.B = Wb + ro.n1_w + kLat; c.ldb = 2 * kLat; c.b_trans = 1;
      c.M = n; c.N = kLat; c.K = kLat;
      c.c_bf16 = s->dm; c.ldc = kLat;
      TRYS(run(s, c));
    }
    TRYS(wgrad(s, s->dm, kLat, kLat, s->S[r], kLat, kLat, n, G + ro.w2));
    {
      GemmCall c;  // dS = dm . W2
      c.A = s->dm; c.lda = kLat; c.B = Wb + ro.w2; c.ldb = kLat; c.b_trans = 1;
      c.M = n; c.N = kLat; c.K = kLat;
      c.c_f32 = s->dS; c.ldc = kLat;
      TRYS(run(s, c));
    }
    k_sur_edge_bwd<<<kEdgeBlocks, kEdgeThreads, 0, q>>>(n, s->PQ[r], s->w + ro.we, s->nbr, s->ef, s->deg, s->dS,
                                                        s->dPQ, s->wepart);
    sum_rows(s->wepart, kEdgeBlocks, kLat * 4, G + ro.we, q);
    TRYS(wgrad(s, s->dPQ, 2 * kLat, 2 * kLat, s->cat[r], 2 * kLat, kLat, n, G + ro.pq_w));
    TRYS(colsum(s, s->dPQ, 2 * kLat, 2 * kLat, n, G + ro.pq_b));
    {
      GemmCall c;  // dh += dPQ . W_pq
      c.A = s->dPQ; c.lda = 2 * kLat; c.B = Wb + ro.pq_w; c.ldb = kLat; c.b_trans = 1;
      c.M = n; c.N = kLat; c.K = 2 * kLat;
      c.accumulate = 1; c.c_f32 = s->dh; c.ldc = kLat;
      TRYS(run(s, c));
    }
  }
  k_f32_to_bf16<<<(unsigned)((nl + 255) / 256), 256, 0, q>>>(s->dh, s->dhb, nl);
  TRYS(wgrad(s, s->dhb, kLat, kLat, s->a1, kLat, kLat, n, G + o.enc2_w));
  TRYS(colsum(s, s->dhb, kLat, kLat, n, G + o.enc2_b));
  {
    GemmCall c;  // dz = (dh . Enc2) masked by a1 > 0
    c.A = s->dhb; c.lda = kLat; c.B = Wb + o.enc2_w; c.ldb = kLat; c.b_trans = 1;
    c.M = n; c.N = kLat; c.K = kLat;
    c.mask = s->a1; c.ldm = kLat; c.c_bf16 = s->dz; c.ldc = kLat;
    TRYS(run(s, c));
  }
  TRYS(wgrad(s, s->dz, kLat, kLat, s->F, kFeat, kFeat, n, G + o.enc1_w));
  TRYS(colsum(s, s->dz, kLat, kLat, n, G + o.enc1_b));
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

NodesView view_of(const uph_sur_nodes *nd)
{
  NodesView v;
  v.n = nd->n;
  v.nf = nd->n_fluid;
  v.x = nd->x;
  v.y = nd->y;
  v.u = nd->u;
  v.v = nd->v;
  v.rho = nd->rho;
  v.itype = nd->itype;
  v.lo_x = nd->lo_x;
  v.lo_y = nd->lo_y;
  v.hi_x = nd->hi_x;
  v.hi_y = nd->hi_y;
  return v;
}

bool nodes_ok(const uph_sur_nodes *nd)
{
  return nd && nd->x && nd->y && nd->u && nd->v && nd->rho && nd->itype;
}

}  // namespace

// ---- C ABI ------------------------------------------------------------------------
extern "C" int64_t uph_sur_param_count(int32_t rounds)
{
  if (rounds < 1 || rounds > kMaxRounds) return -1;
  return (int64_t)param_layout(rounds).total;
}

extern "C" uph_status uph_sur_create(const uph_sur_config *cfg, int32_t node_capacity, uph_surrogate **out)
{
  if (!cfg || !out) return fail(UPH_BAD_ARG, "uph_sur_create: NULL argument");
  *out = nullptr;
  if (cfg->rounds < 1 || cfg->rounds > kMaxRounds) return fail(UPH_BAD_ARG, "uph_sur_create: rounds outside 1..4");
  if (!(cfg->radius > 0.0) || !(cfg->dt > 0.0) || !(cfg->rho0 > 0.0) || !(cfg->vel_scale > 0.0) ||
      !(cfg->rho_scale > 0.0) || !(cfg->edge_rho_scale > 0.0) || cfg->macro_steps < 1)
    return fail(UPH_BAD_ARG, "uph_sur_create: radius, dt, rho0, scales and macro_steps must be positive");
  if (node_capacity < 1 || node_capacity > (1 << 26)) return fail(UPH_BAD_ARG, "uph_sur_create: bad node capacity");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(UPH_NO_DEVICE, "uph_sur_create: no CUDA device");
  uph_surrogate *s = new uph_surrogate();
  s->cfg = *cfg;
  s->off = param_layout(cfg->rounds);
  s->cap = (node_capacity + 127) / 128 * 128;
  const size_t c = (size_t)s->cap;
  const size_t P = s->off.total;
  cudaError_t e = cudaSuccess;
  auto A = [&](auto **p, size_t count) {
    if (e == cudaSuccess) e = salloc(s, p, count);
  };
  A(&s->d_err, 1);
  A(&s->d_bad, 1);
  A(&s->w, P);
  A(&s->g, P);
  A(&s->am, P);
  A(&s->av, P);
  A(&s->wb, P);
  A(&s->nbr, c * kMaxDeg);
  A(&s->ef, c * kMaxDeg);
  A(&s->deg, c);
  A(&s->grid.list, c);
  A(&s->grid.cell_of, c);
  A(&s->F, c * kFeat);
  A(&s->a1, c * kLat);
  A(&s->d1, c * kLat);
  A(&s->out, c * kOutPad);
  for (int r = 0; r <= cfg->rounds; r++) A(&s->cat[r], c * 2 * kLat);
  for (int r = 0; r < cfg->rounds; r++) {
    A(&s->PQ[r], c * 2 * kLat);
    A(&s->S[r], c * kLat);
    A(&s->u[r], c * kLat);
  }
  A(&s->dO, c * kOutPad);
  A(&s->dz, c * kLat);
  A(&s->dhb, c * kLat);
  A(&s->dm, c * kLat);
  A(&s->dPQ, c * 2 * kLat);
  A(&s->dh, c * kLat);
  A(&s->dS, c * kLat);
  A(&s->partials, (size_t)kSplitMax * 128 * 128);
  A(&s->colpart, (size_t)kColBlocks * 2 * kLat);
  A(&s->wepart, (size_t)kEdgeBlocks * kLat * 4);
  A(&s->losspart, kLossBlocks);
  A(&s->lossval, 1);
  A(&s->sqpart, 296);
  A(&s->sumsq, 1);
  A(&s->jpart, 2 * kJudgeBlocks);
  A(&s->wimg, P * sizeof(bf16));
  A(&s->hb[0], c * kLat);
  A(&s->hb[1], c * kLat);
  A(&s->bins, 2 * kMaxBins);
  if (e != cudaSuccess) {
    free_all(s);
    delete s;
    return e == cudaErrorMemoryAllocation ? fail(UPH_OUT_OF_MEMORY, "uph_sur_create: out of device memory")
                                          : cuda_fail(e, "cudaMalloc");
  }
  uph_status tr = make_row_tensor_map(&s->tm_F, s->F, s->cap, kFeat, kFeat * 2);
  if (tr == UPH_OK) tr = make_row_tensor_map(&s->tm_S, s->S[0], s->cap, kLat, kLat * 2);
  if (tr == UPH_OK) tr = make_row_tensor_map(&s->tm_PQ, s->PQ[0], s->cap, 2 * kLat, 2 * kLat * 2);
  for (int k = 0; k < 2 && tr == UPH_OK; k++) tr = make_row_tensor_map(&s->tm_H[k], s->hb[k], s->cap, kLat, kLat * 2);
  if (tr != UPH_OK) {
    free_all(s);
    delete s;
    return tr;
  }
  cudaMemset(s->d_err, 0, sizeof(unsigned));
  cudaMemset(s->w, 0, sizeof(float) * P);
  cudaMemset(s->wb, 0, sizeof(bf16) * P);
  cudaMemset(s->am, 0, sizeof(float) * P);
  cudaMemset(s->av, 0, sizeof(float) * P);
  const cudaError_t me = cudaDeviceSynchronize();
  if (me != cudaSuccess) {
    free_all(s);
    delete s;
    return cuda_fail(me, "uph_sur_create");
  }
  *out = s;
  return UPH_OK;
}

extern "C" uph_status uph_sur_destroy(uph_surrogate *s)
{
  if (!s) return UPH_OK;
  cudaStreamSynchronize(s->stream);
  for (void *p : {(void *)s->grid.count, (void *)s->grid.start, (void *)s->grid.fill, (void *)s->grid.block_sums,
                  (void *)s->pred})
    if (p) cudaFree(p);
  free_all(s);
  delete s;
  return UPH_OK;
}

extern "C" uph_status uph_sur_set_stream(uph_surrogate *s, void *stream)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL surrogate");
  s->stream = (cudaStream_t)stream;
  return UPH_OK;
}

extern "C" uph_status uph_sur_set_params(uph_surrogate *s, const float *host, int64_t count)
{
  if (!s || !host) return fail(UPH_BAD_ARG, "uph_sur_set_params: NULL argument");
  if (count != (int64_t)s->off.total) return fail(UPH_BAD_ARG, "uph_sur_set_params: wrong parameter count");
  UPH_CUDA(cudaMemcpyAsync(s->w, host, sizeof(float) * count, cudaMemcpyHostToDevice, s->stream));
  k_f32_to_bf16<<<(unsigned)((count + 255) / 256), 256, 0, s->stream>>>(s->w, s->wb, (size_t)count);
  s->img_dirty = true;
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

extern "C" uph_status uph_sur_get_params(uph_surrogate *s, float *host, int64_t count)
{
  if (!s || !host) return fail(UPH_BAD_ARG, "uph_sur_get_params: NULL argument");
  if (count != (int64_t)s->off.total) return fail(UPH_BAD_ARG, "uph_sur_get_params: wrong parameter count");
  UPH_CUDA(cudaMemcpyAsync(host, s->w, sizeof(float) * count, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  return UPH_OK;
}

extern "C" uph_status uph_sur_set_fused(uph_surrogate *s, int32_t on)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL surrogate");
  s->fused = on != 0;
  return UPH_OK;
}

extern "C" uph_status uph_sur_reset_optimizer(uph_surrogate *s)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL surrogate");
  UPH_CUDA(cudaMemsetAsync(s->am, 0, sizeof(float) * s->off.total, s->stream));
  UPH_CUDA(cudaMemsetAsync(s->av, 0, sizeof(float) * s->off.total, s->stream));
  s->adam_t = 0;
  return UPH_OK;
}

extern "C" uph_status uph_sur_forward(uph_surrogate *s, const uph_sur_nodes *nodes, float *out)
{
  if (!s || !nodes_ok(nodes)) return fail(UPH_BAD_ARG, "uph_sur_forward: NULL argument");
  const NodesView nv = view_of(nodes);
  TRYS(prepare(s, nv));
  TRYS(forward_any(s, nv.n));
  if (out) k_copy_out<<<(nv.n * kNOut + 255) / 256, 256, 0, s->stream>>>(nv.n, s->out, out);
  s->n_last = nv.n;
  s->nf_last = nv.nf;
  TRYS(check_err(s));
  return UPH_OK;
}

extern "C" uph_status uph_sur_gradients(uph_surrogate *s, const uph_sur_nodes *nodes, const float *target, float *grad,
                                        double *loss)
{
  if (!s || !nodes_ok(nodes) || !target) return fail(UPH_BAD_ARG, "uph_sur_gradients: NULL argument");
  const NodesView nv = view_of(nodes);
  if (nv.nf < 1) return fail(UPH_BAD_ARG, "uph_sur_gradients: no fluid nodes");
  TRYS(prepare(s, nv));
  TRYS(forward_net(s, nv.n));
  const float inv_count = 1.0f / (float)((double)nv.nf * kNOut);
  k_sur_loss<<<kLossBlocks, 256, 0, s->stream>>>(nv.n, nv.nf, s->out, target, inv_count, s->dO, s->losspart);
  sum_rows(s->losspart, kLossBlocks, 1, s->lossval, s->stream);
  TRYS(backward_net(s, nv.n));
  if (grad)
    UPH_CUDA(cudaMemcpyAsync(grad, s->g, sizeof(float) * s->off.total, cudaMemcpyDeviceToDevice, s->stream));
  s->have_grad = true;
  s->n_last = nv.n;
  s->nf_last = nv.nf;
  if (loss) {
    float l = 0.0f;
    UPH_CUDA(cudaMemcpyAsync(&l, s->lossval, sizeof l, cudaMemcpyDeviceToHost, s->stream));
    TRYS(check_err(s));
    *loss = l;
  }
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

extern "C" uph_status uph_sur_adam(uph_surrogate *s, double lr, double beta1, double beta2, double eps, double clip)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL surrogate");
  if (!s->have_grad) return fail(UPH_BAD_ARG, "uph_sur_adam: no gradients computed yet");
  if (!(lr > 0.0) || !(beta1 >= 0.0 && beta1 < 1.0) || !(beta2 >= 0.0 && beta2 < 1.0) || !(eps > 0.0))
    return fail(UPH_BAD_ARG, "uph_sur_adam: bad hyper-parameters");
  const size_t P = s->off.total;
  s->adam_t++;
  const double c1 = 1.0 / (1.0 - pow(beta1, s->adam_t)), c2 = 1.0 / (1.0 - pow(beta2, s->adam_t));
  if (clip > 0.0) {
    k_sumsq_part<<<296, 256, 0, s->stream>>>(s->g, P, s->sqpart);
    sum_rows(s->sqpart, 296, 1, s->sumsq, s->stream);
  }
  k_adam<<<(unsigned)((P + 255) / 256), 256, 0, s->stream>>>(P, s->w, s->g, s->am, s->av, s->wb, (float)lr,
                                                              (float)beta1, (float)beta2, (float)eps, (float)c1,
                                                              (float)c2, s->sumsq, (float)clip);
  s->img_dirty = true;
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

namespace {

// graph and features of the simulation's current state (no synchronisation:
// a node with too many partners is found with the prediction's guard)
uph_status prepare_sim(uph_surrogate *s, uph_sim *sim)
{
  SimView sv = sim_view(sim);
  if (s->cap < sv.P.n) return fail(UPH_BAD_ARG, "uph_sur_advance: simulation larger than the node capacity");
  NodesView nv;
  nv.n = sv.P.n;
  nv.nf = sv.P.nf;
  nv.x = sv.S.x;
  nv.y = sv.S.y;
  nv.u = sv.S.u;
  nv.v = sv.S.v;
  nv.rho = sv.S.rho;
  nv.itype = sv.S.itype;
  nv.lo_x = sv.P.lo_x;
  nv.lo_y = sv.P.lo_y;
  nv.hi_x = sv.P.hi_x;
  nv.hi_y = sv.P.hi_y;
  return prepare(s, nv);
}

// the prepared graph through the network into s->pred, then one
// synchronisation for both checks: *fits is false when a node had more
// partners than the graph holds (the flag is cleared; the prediction is not
// to be used), *ok false when the sanity guard rejects the prediction
uph_status network_predict(uph_surrogate *s, uph_sim *sim, bool *fits, bool *ok)
{
  SimView sv = sim_view(sim);
  TRYS(forward_any(s, sv.P.n));
  OutScale sc;
  sc.T = s->cfg.macro_steps * s->cfg.dt;
  for (int k = 0; k < kNOut; k++) sc.s[k] = s->cfg.out_scale[k];
  sc.max_move = s->cfg.radius;
  sc.min_gap = 0.25 * s->cfg.radius;
  UPH_CUDA(cudaMemsetAsync(s->d_bad, 0, sizeof(unsigned), s->stream));
  if (sv.P.nf > 0)
    k_sur_predict<<<(sv.P.nf + 255) / 256, 256, 0, s->stream>>>(sv.P, sv.S, s->out, sc, s->nbr, s->deg, s->pred,
                                                                 s->d_bad);
  unsigned bad = 0, err = 0;
  UPH_CUDA(cudaMemcpyAsync(&bad, s->d_bad, sizeof bad, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof err, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  UPH_CUDA(cudaGetLastError());
  *fits = !(err & ERR_NEIGHBOR_OVERFLOW);
  if (!*fits) {
    err &= ~ERR_NEIGHBOR_OVERFLOW;
    UPH_CUDA(cudaMemcpyAsync(s->d_err, &err, sizeof err, cudaMemcpyHostToDevice, s->stream));
  }
  if (err) return check_err(s);
  *ok = bad == 0;
  return UPH_OK;
}

// s->pred becomes the simulation's fluid state, `nsteps` SPH steps after
// the current time (0 when the plain solver already advanced the clock)
uph_status network_commit(uph_surrogate *s, uph_sim *sim, int nsteps)
{
  SimView sv = sim_view(sim);
  if (sv.P.nf > 0) k_sur_commit<<<(sv.P.nf + 255) / 256, 256, 0, s->stream>>>(sv.P, sv.S, s->pred);
  UPH_CUDA(cudaGetLastError());
  return sim_jump(sim, nsteps);
}

}  // namespace

extern "C" uph_status uph_sur_advance(uph_surrogate *s, uph_sim *sim, int32_t macro_steps, const uph_sur_judge *judge,
                                      uph_sur_report *report)
{
  if (!s || !sim || !judge || !report) return fail(UPH_BAD_ARG, "uph_sur_advance: NULL argument");
  if (macro_steps < 0) return fail(UPH_BAD_ARG, "uph_sur_advance: negative step count");
  if (judge->judge_every < 1 || judge->fallback_macro < 0 || judge->surface_bins < 1 ||
      judge->surface_bins > kMaxBins || !(judge->surface_x1 > judge->surface_x0) || !(judge->depth > 0.0))
    return fail(UPH_BAD_ARG, "uph_sur_advance: bad judge settings");
  SimView sv = sim_view(sim);
  // the network runs on the simulation's stream for the whole call
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  struct StreamSwap {
    uph_surrogate *s;
    cudaStream_t saved;
    ~StreamSwap() { s->stream = saved; }
  } swap{s, s->stream};
  s->stream = sv.stream;
  if (sv.P.profile != UPH_PROFILE_WCSPH)
    return fail(UPH_UNSUPPORTED, "uph_sur_advance: the surrogate advances WCSPH simulations only");
  if (fabs(sv.P.dt - s->cfg.dt) > 1e-12 * s->cfg.dt)
    return fail(UPH_BAD_ARG, "uph_sur_advance: the simulation's dt differs from the network's");
  const int K = s->cfg.macro_steps;
  if (sv.serial != s->last_sim) {
    s->last_sim = sv.serial;
    s->since_judge = 0;
    s->fallback_left = 0;
  }
  // the judge's prediction buffer: reference-indexed so it survives re-sorts
  if (!s->pred || s->n_pred < sv.P.nf) {
    if (s->pred) cudaFree(s->pred);
    s->pred = nullptr;
    s->n_pred = 0;
    UPH_CUDA(cudaMalloc((void **)&s->pred, sizeof(double) * kNOut * (size_t)std::max(sv.P.nf, 1)));
    s->n_pred = sv.P.nf;
  }
  for (int m = 0; m < macro_steps; m++) {
    report->macro_steps++;
    if (s->fallback_left > 0) {
      s->fallback_left--;
      TRYS(uph_sim_step(sim, K));
      report->plain_steps += K;
      continue;
    }
    s->since_judge++;
    bool fits = true, ok = true;
    TRYS(prepare_sim(s, sim));
    TRYS(network_predict(s, sim, &fits, &ok));
    if (!fits) {
      // a state the network's graph cannot hold: the plain solver takes
      // this macro step and the fallback after it
      report->graph_overflows++;
      s->since_judge = 0;
      s->fallback_left = judge->fallback_macro;
      TRYS(uph_sim_step(sim, K));
      report->plain_steps += K;
      continue;
    }
    if (!ok) {
      // an implausible prediction (non-finite, or density beyond the guard
      // band) never reaches the state: the plain solver takes over
      report->rejected_steps++;
      s->since_judge = 0;
      s->fallback_left = judge->fallback_macro;
      TRYS(uph_sim_step(sim, K));
      report->plain_steps += K;
      continue;
    }
    if (s->since_judge < judge->judge_every) {
      TRYS(network_commit(s, sim, K));
      report->network_steps++;
      continue;
    }
    // judged macro step: the plain solver runs over the same span from the
    // same state; a prediction that passes the check is kept (the network's
    // trajectory goes on undisturbed), a failed one leaves the plain state
    // and starts the fallback
    s->since_judge = 0;
    TRYS(uph_sim_step(sim, K));
    report->plain_steps += K;
    report->judged_steps++;
    sv = sim_view(sim);
    const int nb = judge->surface_bins;
    UPH_CUDA(cudaMemsetAsync(s->bins, 0, sizeof(unsigned) * 2 * nb, s->stream));
    k_sur_judge<<<kJudgeBlocks, 256, 0, s->stream>>>(sv.P, sv.S, s->pred, judge->surface_x0,
                                                     nb / (judge->surface_x1 - judge->surface_x0), nb, s->bins,
                                                     s->bins + nb, s->jpart);
    std::vector<double> part(2 * kJudgeBlocks);
    std::vector<unsigned> bins(2 * nb);
    UPH_CUDA(cudaMemcpyAsync(part.data(), s->jpart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s->stream));
    UPH_CUDA(cudaMemcpyAsync(bins.data(), s->bins, sizeof(unsigned) * bins.size(), cudaMemcpyDeviceToHost, s->stream));
    TRYS(check_err(s));
    double sq = 0.0;
    for (int b = 0; b < kJudgeBlocks; b++) sq += part[2 * b];
    const double rho_err = sv.P.nf > 0 ? sqrt(sq / sv.P.nf) : 0.0;
    double surf = 0.0;
    for (int b = 0; b < nb; b++) {
      if (!bins[b] || !bins[nb + b]) continue;  // a bin empty in either state
      auto val = [](unsigned o) {
        const unsigned bits = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
        float f;
        memcpy(&f, &bits, sizeof f);
        return (double)f;
      };
      surf = std::max(surf, fabs(val(bins[nb + b]) - val(bins[b])) / judge->depth);
    }
    report->last_rho_err = rho_err;
    report->last_surface_err = surf;
    report->max_rho_err = std::max(report->max_rho_err, rho_err);
    report->max_surface_err = std::max(report->max_surface_err, surf);
    if (!(rho_err <= judge->max_rho_err) || !(surf <= judge->max_surface_err)) {
      report->failed_checks++;
      s->fallback_left = judge->fallback_macro;
    } else {
      TRYS(network_commit(s, sim, 0));
      report->network_steps++;
    }
  }
  return sim_check(sim);
}
