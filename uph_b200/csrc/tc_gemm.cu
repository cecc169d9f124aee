// BF16 tensor-core GEMM on sm_100a (tcgen05), FP32 accumulation in TMEM.
//
//   C[M x N] = A[M x K] . B[N x K]^T  (+ bias[N], optional ReLU)
//
// A and B are row-major with K contiguous ("K-major"), K a multiple of 64,
// N a multiple of 128.  One CTA of 128 threads computes a 128 x 128 tile of
// C over a K range (the whole K, or one split of it):
//   - the 128 threads copy a 128 x 64 slice of A and of B into shared memory
//     in the 128-byte-swizzled K-major layout that UMMA descriptors describe
//     (16-byte chunk c of row r at r*128 + ((c ^ (r % 8)) * 16) inside a
//     1024-byte-aligned tile), two stages so the next copy overlaps the MMAs;
//   - one thread issues four tcgen05.mma (M = 128, N = 128, K = 16 each,
//     kind::f16 with BF16 inputs) into a 128-column FP32 accumulator in TMEM
//     and commits them to an mbarrier;
//   - after the last slice, each warp reads its 32 TMEM lanes (one output row
//     per thread) with tcgen05.ld and applies the epilogue.
// Split-K launches write FP32 partial tiles that k_splitk_reduce sums in a
// fixed order (deterministic).
//
// Every mbarrier wait is bounded; a wait that gives up sets ERR_TIMEOUT in the
// error word, and the CTA still frees its TMEM before returning.
#include <cuda_bf16.h>

#include <cute/arch/mma_sm100_desc.hpp>
#include <cute/numeric/numeric_types.hpp>

#include "uph_internal.cuh"
#include "uph_surrogate.h"

namespace uph {

constexpr int kTcM = 128;       // rows of C per CTA (UMMA M)
constexpr int kTcN = 128;       // columns of C per CTA (UMMA N)
constexpr int kTcBK = 64;       // K per shared-memory slice: one 128-byte swizzle atom row
constexpr int kTcUmmaK = 16;    // K of one tcgen05.mma of kind::f16
constexpr int kTcStages = 2;
constexpr int kTcTileBytes = kTcM * kTcBK * 2;  // 16 KiB, same for the B slice (kTcN rows)
constexpr int kTcSmemBytes = kTcStages * 2 * kTcTileBytes + 1024 + 64;
constexpr long long kWaitLimit = 1LL << 26;     // poll cap; the time bound is kWaitNs

struct TcGemmArgs {
  const __nv_bfloat16 *A;
  const __nv_bfloat16 *B;
  int lda, ldb;              // elements
  int a_trans, b_trans;      // operand stored as [K x rows] (rows contiguous) instead of [rows x K]
  int M, N, K;               // K multiple of 64, N multiple of 128
  int k_valid;               // transposed operands: K rows >= k_valid read as zero
  int k_per_split;           // multiple of 64
  const float *bias;         // [N] or null
  int relu;
  const __nv_bfloat16 *mask; // [M x ldm] or null: zero the result where mask <= 0
  int ldm;
  int accumulate;            // add the result to c_f32's contents
  const __nv_bfloat16 *residual;  // [M x ldr] or null: added after the bias
  int ldr;
  float *c_f32;              // [M x ldc] or null
  __nv_bfloat16 *c_bf16;     // [M x ldc16] or null
  int ldc, ldc16;
  float *partials;           // split-K: [splits][M][N] FP32
  unsigned *err;
  int stall;                 // self-test of the bounded waits (GemmCall::stall)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t smem_addr)
{
  // K-major, 128-byte swizzle: 8-row groups 1024 bytes apart (SBO), unit
  // leading offset, Blackwell descriptor version
  cute::UMMA::SmemDescriptor d;
  d.desc_ = 0;
  d.start_address_ = static_cast<uint16_t>(smem_addr >> 4);
  d.leading_byte_offset_ = 1;
  d.stride_byte_offset_ = 1024 >> 4;
  d.version_ = 1;
  d.base_offset_ = 0;
  d.lbo_mode_ = 0;
  d.layout_type_ = static_cast<uint8_t>(cute::UMMA::LayoutType::SWIZZLE_128B);
  return d.desc_;
}

// true once the barrier's phase `parity` completed; false after kWaitNs on
// the global timer or kWaitLimit polls, whichever comes first
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
  const unsigned long long t0 = global_ns();
  for (long long i = 0; i < kWaitLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 63) == 63 && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

// copies rows [r0, r0 + 128) x cols [k0, k0 + 64) of a row-major BF16 matrix
// into the swizzled tile at `tile`; rows beyond `rows` read as zero
__device__ __forceinline__ void load_tile(uint8_t *tile, const __nv_bfloat16 *src, int ld, int r0, int rows, int k0)
{
  const int t = threadIdx.x;
  const int c = t & 7;  // 16-byte chunk of the row
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int r = (t >> 3) + 16 * i;
    const int gr = r0 + r;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (gr < rows) v = *reinterpret_cast<const uint4 *>(src + (size_t)gr * ld + k0 + c * 8);
    *reinterpret_cast<uint4 *>(tile + r * 128 + ((c ^ (r & 7)) << 4)) = v;
  }
}

// the same tile from an operand stored transposed, [K x rows] with rows
// contiguous (e.g. node activations [nodes x features] as the K-major operand
// of a weight gradient): a lane loads 8 consecutive rows of one K index and
// stores them one element at a time; the 32 lanes of a warp take 32
// consecutive K, so their stores fall in one 64-byte span of a tile row.
// Rows >= `rows` and K >= k_valid read as zero; rows is a multiple of 8.
__device__ __forceinline__ void load_tile_t(uint8_t *tile, const __nv_bfloat16 *src, int ld, int r0, int rows, int k0,
                                            int k_valid)
{
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int q = t + 128 * i;
    const int kk = q & 63;         // K inside the slice
    const int rc = (q >> 6) * 8;   // first of 8 rows
    const int gk = k0 + kk;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (gk < k_valid && r0 + rc < rows) v = *reinterpret_cast<const uint4 *>(src + (size_t)gk * ld + r0 + rc);
    const uint16_t *e = reinterpret_cast<const uint16_t *>(&v);
    const int chunk = kk >> 3, sub = (kk & 7) * 2;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int r = rc + j;
      *reinterpret_cast<uint16_t *>(tile + r * 128 + ((chunk ^ (r & 7)) << 4) + sub) = e[j];
    }
  }
}

__global__ void __launch_bounds__(128) k_tc_gemm(TcGemmArgs g)
{
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t mbar[kTcStages];
  __shared__ uint64_t stall_bar;  // the self-test's barrier: initialised, never arrived at
  __shared__ uint32_t tmem_base_slot;
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int m0 = blockIdx.x * kTcM, n0 = blockIdx.y * kTcN;
  const int kbeg = blockIdx.z * g.k_per_split;
  const int kend = min(g.K, kbeg + g.k_per_split);
  const int nslices = max(0, (kend - kbeg) / kTcBK);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 0) {  // TMEM: 128 FP32 columns for the 128 x 128 accumulator
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                 "r"(kTcN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTcStages; s++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&stall_bar)));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_slot;

  const uint32_t idesc = static_cast<uint32_t>(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, kTcM, kTcN,
                                                                            cute::UMMA::Major::K, cute::UMMA::Major::K>());
  // the self-test waits for a phase that never completes: the bounded wait
  // gives up, no copy or MMA has been issued, and the CTA goes straight to
  // freeing its TMEM
  // Every thread polls on its own clock, so a wait that gives up near the
  // limit can give up in some threads only: each outcome is made uniform
  // over the block before anyone acts on it.
  bool ok = g.stall ? mbar_wait(smem_u32(&stall_bar), 0u) : true;
  ok = __syncthreads_and(ok) != 0;
  int issued = 0;  // slices whose MMAs were issued (and committed to their stage's barrier)
  for (int s = 0; s < nslices && ok; s++) {
    const int st = s % kTcStages;
    uint8_t *ta = smem + st * 2 * kTcTileBytes;
    uint8_t *tb = ta + kTcTileBytes;
    // the stage's previous MMAs must be done before its tiles are overwritten:
    // commit number s / kTcStages - 1 of this stage completes phase parity
    // (s / kTcStages - 1) & 1
    if (s >= kTcStages) {
      ok = mbar_wait(smem_u32(&mbar[st]), (uint32_t)((s / kTcStages - 1) & 1));
      ok = __syncthreads_and(ok) != 0;
      if (!ok) break;
    }
    const int k0 = kbeg + s * kTcBK;
    if (g.a_trans)
      load_tile_t(ta, g.A, g.lda, m0, g.M, k0, g.k_valid);
    else
      load_tile(ta, g.A, g.lda, m0, g.M, k0);
    if (g.b_trans)
      load_tile_t(tb, g.B, g.ldb, n0, g.N, k0, g.k_valid);
    else
      load_tile(tb, g.B, g.ldb, n0, g.N, k0);
    // generic-proxy shared stores -> visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
      const uint32_t a_addr = smem_u32(ta), b_addr = smem_u32(tb);
#pragma unroll
      for (int kk = 0; kk < kTcBK / kTcUmmaK; kk++) {
        // advancing K inside the 128-byte swizzle atom moves the start address
        const uint64_t da = umma_desc_sw128(a_addr + kk * kTcUmmaK * 2);
        const uint64_t db = umma_desc_sw128(b_addr + kk * kTcUmmaK * 2);
        const uint32_t accumulate = (s > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[st]))
                   : "memory");
    }
    issued = s + 1;
  }
  // Drain: wait for the last commit of every stage that was used, on the
  // normal path and after a failed wait alike, so that no MMA still writes
  // the accumulator when TMEM is freed.  A stage with c commits has its last
  // one complete phase parity (c - 1) & 1; waiting on a phase that already
  // completed returns at once.
  bool drained = true;
  for (int st = 0; st < kTcStages; st++) {
    const int c = (issued - st + kTcStages - 1) / kTcStages;
    if (c > 0 && !mbar_wait(smem_u32(&mbar[st]), (uint32_t)((c - 1) & 1))) drained = false;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  drained = __syncthreads_and(drained) != 0;
  ok = ok && drained;

  if (!ok) {
    if (threadIdx.x == 0) atomicOr(g.err, ERR_TIMEOUT);
  } else {
    // epilogue: warp w owns TMEM lanes [32w, 32w + 32) = rows m0 + 32w + lane
    const int row = m0 + warp * 32 + lane;
    const uint32_t lane_addr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
    for (int c0 = 0; c0 < kTcN; c0 += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(lane_addr + c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < g.M && nslices > 0) {
        const int col = n0 + c0;
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
        if (g.partials) {
          float *dst = g.partials + ((size_t)blockIdx.z * g.M + row) * g.N + col;
#pragma unroll
          for (int j = 0; j < 16; j += 4) *reinterpret_cast<float4 *>(dst + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        } else {
          if (g.bias)
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] += g.bias[col + j];
          if (g.residual) {
            const __nv_bfloat16 *rs = g.residual + (size_t)row * g.ldr + col;
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] += __bfloat162float(rs[j]);
          }
          if (g.accumulate) {
            const float *old = g.c_f32 + (size_t)row * g.ldc + col;
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] += old[j];
          }
          if (g.relu)
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] = fmaxf(v[j], 0.0f);
          if (g.mask) {
            const __nv_bfloat16 *mk = g.mask + (size_t)row * g.ldm + col;
#pragma unroll
            for (int j = 0; j < 16; j++)
              if (!(__bfloat162float(mk[j]) > 0.0f)) v[j] = 0.0f;
          }
          if (g.c_f32) {
            float *dst = g.c_f32 + (size_t)row * g.ldc + col;
#pragma unroll
            for (int j = 0; j < 16; j += 4)
              *reinterpret_cast<float4 *>(dst + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
          }
          if (g.c_bf16) {
            __nv_bfloat16 *dst = g.c_bf16 + (size_t)row * g.ldc16 + col;
            __align__(16) __nv_bfloat162 h[8];
#pragma unroll
            for (int j = 0; j < 8; j++) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<uint4 *>(&h[0]);
            *reinterpret_cast<uint4 *>(dst + 8) = *reinterpret_cast<uint4 *>(&h[4]);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // an MMA that never completed may still write the accumulator: its TMEM
  // is then left allocated rather than freed under it (the error word
  // already says the tensor core stopped answering)
  if (warp == 0 && drained)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcN));
}

// out[m][n] (+)= sum over splits of partials[s][m][n], in split order
__global__ void k_splitk_reduce(const float *__restrict__ partials, int splits, int M, int N, float *out,
                                int accumulate)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  float acc = accumulate ? out[i] : 0.0f;
  for (int s = 0; s < splits; s++) acc += partials[(size_t)s * M * N + i];
  out[i] = acc;
}


uph_status launch_tc_gemm(const GemmCall &c, cudaStream_t s)
{
  if (!c.A || !c.B || !c.err || c.M <= 0 || c.N <= 0 || c.K <= 0) return fail(UPH_BAD_ARG, "tc_gemm: bad arguments");
  if (c.K % kTcBK || c.N % kTcN) return fail(UPH_BAD_ARG, "tc_gemm: K must be a multiple of 64, N of 128");
  const int ldc16 = c.ldc16 > 0 ? c.ldc16 : c.ldc;
  if (c.lda % 8 || c.ldb % 8 || c.ldc % 8 || ldc16 % 8 || (c.mask && c.ldm % 8) || (c.residual && c.ldr % 8))
    return fail(UPH_BAD_ARG, "tc_gemm: leading dimensions must be multiples of 8");
  if ((c.a_trans && c.M % 8) || (c.b_trans && c.N % 8))
    return fail(UPH_BAD_ARG, "tc_gemm: a transposed operand needs a multiple of 8 rows");
  int splits = c.splits < 1 ? 1 : c.splits;
  if (splits > 1 && (!c.partials || !c.c_f32 || c.bias || c.relu || c.c_bf16 || c.mask || c.residual || c.ldc != c.N))
    return fail(UPH_BAD_ARG, "tc_gemm: split-K writes a dense FP32 result only, without bias, ReLU or mask");
  if (splits == 1 && !c.c_f32 && !c.c_bf16) return fail(UPH_BAD_ARG, "tc_gemm: no output");
  if (splits == 1 && c.accumulate && !c.c_f32) return fail(UPH_BAD_ARG, "tc_gemm: accumulate needs c_f32");
  static bool configured = false;
  if (!configured) {
    UPH_CUDA(cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemBytes));
    configured = true;
  }
  TcGemmArgs g;
  g.A = (const __nv_bfloat16 *)c.A;
  g.B = (const __nv_bfloat16 *)c.B;
  g.lda = c.lda;
  g.ldb = c.ldb;
  g.a_trans = c.a_trans;
  g.b_trans = c.b_trans;
  g.M = c.M;
  g.N = c.N;
  g.K = c.K;
  g.k_valid = c.k_valid > 0 ? c.k_valid : c.K;
  int kps = c.K;
  if (splits > 1) kps = ((c.K / kTcBK + splits - 1) / splits) * kTcBK;
  g.k_per_split = kps;
  splits = (c.K + kps - 1) / kps;
  g.bias = c.bias;
  g.relu = c.relu;
  g.mask = (const __nv_bfloat16 *)c.mask;
  g.ldm = c.ldm;
  g.accumulate = splits > 1 ? 0 : c.accumulate;
  g.residual = (const __nv_bfloat16 *)c.residual;
  g.ldr = c.ldr;
  g.c_f32 = splits > 1 ? nullptr : c.c_f32;
  g.c_bf16 = (__nv_bfloat16 *)c.c_bf16;
  g.ldc = c.ldc;
  g.ldc16 = ldc16;
  g.partials = splits > 1 ? c.partials : nullptr;
  g.err = c.err;
  g.stall = c.stall;
  dim3 grid((c.M + kTcM - 1) / kTcM, c.N / kTcN, splits);
  k_tc_gemm<<<grid, 128, kTcSmemBytes, s>>>(g);
  if (splits > 1) {
    const int total = c.M * c.N;
    k_splitk_reduce<<<(total + 255) / 256, 256, 0, s>>>(c.partials, splits, c.M, c.N, c.c_f32, c.accumulate);
  }
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

}  // namespace uph

using namespace uph;

// C ABI for tests: device pointers, both operands K-major.  splits > 1
// requires `partials` of splits * M * N floats and writes the sum into c_f32
// (accumulated onto its contents when accumulate != 0).
extern "C" uph_status uph_tc_gemm_bf16(const void *A, int32_t lda, const void *B, int32_t ldb, int32_t M, int32_t N,
                                       int32_t K, const float *bias, int32_t relu, float *c_f32, void *c_bf16,
                                       int32_t ldc, int32_t splits, float *partials, int32_t accumulate,
                                       unsigned *err, void *stream)
{
  GemmCall c;
  c.A = A;
  c.lda = lda;
  c.B = B;
  c.ldb = ldb;
  c.M = M;
  c.N = N;
  c.K = K;
  c.bias = bias;
  c.relu = relu;
  c.c_f32 = c_f32;
  c.c_bf16 = c_bf16;
  c.ldc = ldc;
  c.splits = splits;
  c.partials = partials;
  c.accumulate = accumulate;
  c.err = err;
  return launch_tc_gemm(c, (cudaStream_t)stream);
}

// Failure-detection self test: one tile whose CTA waits on a barrier nothing
// arrives at.  The bounded wait gives up, the kernel sets ERR_TIMEOUT, frees
// its TMEM and returns; the context stays usable.
extern "C" uph_status uph_tc_wait_selftest(const void *A, const void *B, float *c_f32, unsigned *err, void *stream)
{
  if (!A || !B || !c_f32 || !err) return fail(UPH_BAD_ARG, "uph_tc_wait_selftest: NULL argument");
  cudaStream_t q = (cudaStream_t)stream;
  GemmCall c;
  c.A = A;
  c.lda = kTcBK;
  c.B = B;
  c.ldb = kTcBK;
  c.M = kTcM;
  c.N = kTcN;
  c.K = kTcBK;
  c.c_f32 = c_f32;
  c.ldc = kTcN;
  c.err = err;
  c.stall = 1;
  UPH_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), q));
  uph_status r = launch_tc_gemm(c, q);
  if (r != UPH_OK) return r;
  unsigned e = 0;
  UPH_CUDA(cudaMemcpyAsync(&e, err, sizeof e, cudaMemcpyDeviceToHost, q));
  UPH_CUDA(cudaStreamSynchronize(q));
  if (e & ERR_TIMEOUT) return fail(UPH_TIMEOUT, "uph_tc_wait_selftest: the wait gave up as intended");
  return UPH_OK;
}
