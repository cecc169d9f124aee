// Fused node-side layers of the surrogate network on the tcgen05 tensor cores.
//
// Between two edge layers every layer of the network is node-local, so a
// 128-row tile of nodes can run through all of them without leaving the SM:
//   encoder: F -> relu(E1 F + b) -> h0 = E2 (.) + b -> [P | Q] = W_pq h0 + b
//   round:   S, h -> m = W2 S -> u = relu(N1 [h ; m] + b) -> h' = h + N2 u + b
//            -> [P | Q]' = W_pq' h' + b        (or, in the last round,
//            -> relu(Dec1 h' + b) -> out = Dec2 (.) + b)
// Each CTA (one per SM, persistent over tiles) keeps in shared memory
//   A    2 atoms   the tile's first operand (F or S) and later hidden layers
//   CAT  4 atoms   [h | m] as the K = 256 operand of N1
//   W0/W1          two weight slots of 64 KiB
// (an atom = 128 rows x 64 BF16 columns in the 128-byte-swizzled K-major
// layout of the UMMA descriptors).  Input tiles arrive by TMA (2-D tensor
// maps with 128-byte swizzle, no multicast), weights as pre-swizzled images
// by bulk copies, both completing on mbarriers; each weight is fetched two
// layers ahead, the next tile's inputs as soon as their buffer is free.  One
// thread issues the MMAs (M = 128, N = 128 or 256, K = 16 per instruction)
// into a 256-column TMEM accumulator; after each layer the four warps read
// their 32 TMEM lanes (one row per thread), apply bias / residual / ReLU and
// write the BF16 result into shared memory for the next layer and, where
// needed, to global memory.  Only h, [P | Q] (or the outputs) reach HBM.
//
// The arithmetic is that of the unfused path (tc_gemm.cu) step for step --
// the same K order of MMAs, FP32 bias then residual, the same BF16 rounding
// points -- so both give the same network.
//
// Every mbarrier wait is bounded; a wait that gives up sets ERR_TIMEOUT, the
// CTA stops, waits (bounded) for its copies and MMAs in flight, frees its
// TMEM and returns.
#include <cudaTypedefs.h>

#include <cute/arch/mma_sm100_desc.hpp>
#include <cute/numeric/numeric_types.hpp>

#include "node_chain.cuh"

namespace uph {
namespace {

constexpr int kAtom = 16384;          // 128 rows x 128 bytes
constexpr int kOffA = 0;              // 2 atoms
constexpr int kOffCat = 2 * kAtom;    // 4 atoms: h (atoms 0, 1) | m (atoms 2, 3)
constexpr int kOffW0 = 6 * kAtom;   // weight slot 0 (<= 64 KiB); slot 1 follows
constexpr int kSlotBytes = 4 * kAtom;
constexpr int kSmemUsed = 14 * kAtom; // 224 KiB
constexpr int kSmemBytes = kSmemUsed + 1024;
constexpr int kThreads = 128;
constexpr long long kWaitLimit = 1LL << 26;

struct Shape {
  int n, k;
};

__host__ __device__ inline int layer_count(int mode) { return mode == CHAIN_ENCODER ? 3 : mode == CHAIN_ROUND ? 4 : 5; }

__host__ __device__ inline Shape layer_shape(int mode, int i)
{
  if (mode == CHAIN_ENCODER) return i == 2 ? Shape{256, 128} : Shape{128, 128};
  if (i == 1) return Shape{128, 256};
  if (mode == CHAIN_ROUND && i == 3) return Shape{256, 128};
  return Shape{128, 128};
}

__device__ __forceinline__ uint32_t su32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr)
{
  cute::UMMA::SmemDescriptor d;
  d.desc_ = 0;
  d.start_address_ = static_cast<uint16_t>(addr >> 4);
  d.leading_byte_offset_ = 1;
  d.stride_byte_offset_ = 1024 >> 4;
  d.version_ = 1;
  d.base_offset_ = 0;
  d.lbo_mode_ = 0;
  d.layout_type_ = static_cast<uint8_t>(cute::UMMA::LayoutType::SWIZZLE_128B);
  return d.desc_;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
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
  }
  return false;
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// one 128-row x 64-column box of a 2-D tensor map (x = column, y = row)
__device__ __forceinline__ void tma_load_box(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// C (TMEM) = A (128-row atoms) . B^T (N-row atoms), K / 16 instructions,
// committed to `bar`
__device__ __forceinline__ void issue_mma(uint32_t tmem, uint32_t a, uint32_t b, Shape sh, uint32_t idesc,
                                          uint32_t bar)
{
  for (int ka = 0; ka < sh.k / 64; ka++)
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const uint64_t da = desc_sw128(a + ka * kAtom + kk * 32);
      const uint64_t db = desc_sw128(b + ka * sh.n * 128 + kk * 32);
      const uint32_t acc = (ka | kk) ? 1u : 0u;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
          "l"(da), "l"(db), "r"(idesc), "r"(acc));
    }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float v[16])
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// row r, columns [c0, c0 + 16) of a swizzled K-major buffer of 128-row atoms
__device__ __forceinline__ void smem_put16(uint8_t *buf, int r, int c0, const float v[16])
{
  __align__(16) __nv_bfloat162 h[8];
#pragma unroll
  for (int j = 0; j < 8; j++) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
  uint8_t *row = buf + (c0 >> 6) * kAtom + r * 128;
  const int q = (c0 & 63) >> 3;
  *reinterpret_cast<uint4 *>(row + ((q ^ (r & 7)) << 4)) = *reinterpret_cast<uint4 *>(&h[0]);
  *reinterpret_cast<uint4 *>(row + (((q + 1) ^ (r & 7)) << 4)) = *reinterpret_cast<uint4 *>(&h[4]);
}

__device__ __forceinline__ void smem_get16(const uint8_t *buf, int r, int c0, float v[16])
{
  const uint8_t *row = buf + (c0 >> 6) * kAtom + r * 128;
  const int q = (c0 & 63) >> 3;
  __align__(16) __nv_bfloat162 h[8];
  *reinterpret_cast<uint4 *>(&h[0]) = *reinterpret_cast<const uint4 *>(row + ((q ^ (r & 7)) << 4));
  *reinterpret_cast<uint4 *>(&h[4]) = *reinterpret_cast<const uint4 *>(row + (((q + 1) ^ (r & 7)) << 4));
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const float2 f = __bfloat1622float2(h[j]);
    v[2 * j] = f.x;
    v[2 * j + 1] = f.y;
  }
}

__device__ __forceinline__ void global_put16(__nv_bfloat16 *dst, const float v[16])
{
  __align__(16) __nv_bfloat162 h[8];
#pragma unroll
  for (int j = 0; j < 8; j++) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
  reinterpret_cast<uint4 *>(dst)[0] = *reinterpret_cast<uint4 *>(&h[0]);
  reinterpret_cast<uint4 *>(dst)[1] = *reinterpret_cast<uint4 *>(&h[4]);
}

// what an epilogue does with the accumulator of one layer
enum Epi : int {
  EPI_SMEM = 0,      // (+ bias) (ReLU) -> BF16 into a shared buffer
  EPI_RESIDUAL = 1,  // + bias + h (CAT) -> BF16 into CAT's h and h_out
  EPI_PQ = 2,        // + bias -> BF16 to pq_out (256 columns)
  EPI_OUT = 3,       // + bias -> FP32 to out, columns 0..15
};

struct Step {
  int a_off;   // shared offset of the A operand
  int epi;
  int dst;     // EPI_SMEM: shared offset of the destination
  int relu;
  int h_global;  // EPI_SMEM: also write to h_out (encoder h0)
};

__device__ __forceinline__ Step step_of(int mode, int i)
{
  if (mode == CHAIN_ENCODER) {
    if (i == 0) return Step{kOffA, EPI_SMEM, kOffA, 1, 0};
    if (i == 1) return Step{kOffA, EPI_SMEM, kOffCat, 0, 1};
    return Step{kOffCat, EPI_PQ, 0, 0, 0};
  }
  if (i == 0) return Step{kOffA, EPI_SMEM, kOffCat + 2 * kAtom, 0, 0};
  if (i == 1) return Step{kOffCat, EPI_SMEM, kOffA, 1, 0};
  if (i == 2) return Step{kOffA, EPI_RESIDUAL, 0, 0, 0};
  if (mode == CHAIN_ROUND) return Step{kOffCat, EPI_PQ, 0, 0, 0};
  if (i == 3) return Step{kOffCat, EPI_SMEM, kOffA, 1, 0};
  return Step{kOffA, EPI_OUT, 0, 0, 0};
}

__global__ void __launch_bounds__(kThreads, 1) k_node_chain(const __grid_constant__ ChainArgs a)
{
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[5];  // A tile, h tile, weight slot 0, weight slot 1, MMA
  __shared__ uint32_t tmem_slot;
  __shared__ int s_abort;
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = su32(sm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = warp * 32 + lane;  // tile row = TMEM lane of this thread
  const int L = layer_count(a.mode);
  const bool has_h = a.mode != CHAIN_ENCODER;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_slot)), "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int b = 0; b < 5; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t bar_a = su32(&bars[0]), bar_h = su32(&bars[1]), bar_m = su32(&bars[4]);
  const uint32_t bar_w[2] = {su32(&bars[2]), su32(&bars[3])};
  const uint32_t id128 = static_cast<uint32_t>(
      cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 128, cute::UMMA::Major::K,
                                  cute::UMMA::Major::K>());
  const uint32_t id256 = static_cast<uint32_t>(
      cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 256, cute::UMMA::Major::K,
                                  cute::UMMA::Major::K>());

  // phases of the barriers this thread waits on; thread 0 also keeps the
  // producer's view (and what it has issued but not yet seen complete)
  uint32_t ph_m = 0, ph_h_all = 0;
  uint32_t ph_a = 0, ph_h = 0, ph_w[2] = {0u, 0u};
  bool pend_a = false, pend_h = false, pend_w[2] = {false, false}, pend_m = false;
  const int stride = gridDim.x;
  const int first_tile = blockIdx.x;

  auto tile_of = [&](int it) { return first_tile + it * stride; };
  auto fail_wait = [&]() {
    s_abort = 1;
    atomicOr(a.err, ERR_TIMEOUT);
  };
  // thread 0 only: the weight with global index g (layer g % L of iteration g / L)
  auto issue_weight = [&](int g) {
    const int it = g / L, li = g % L;
    if (tile_of(it) >= a.ntiles) return;
    const Shape sh = layer_shape(a.mode, li);
    const int slot = g & 1;
    const uint32_t bytes = sh.n * sh.k * 2;
    mbar_expect(bar_w[slot], bytes);
    for (uint32_t o = 0; o < bytes; o += kAtom) bulk_load(sb + kOffW0 + slot * kSlotBytes + o, a.layer[li].img + o, kAtom, bar_w[slot]);
    pend_w[slot] = true;
  };
  auto issue_a = [&](int tile) {
    mbar_expect(bar_a, 2 * kAtom);
    tma_load_box(sb + kOffA, &a.tm_a, 0, tile * 128, bar_a);
    tma_load_box(sb + kOffA + kAtom, &a.tm_a, 64, tile * 128, bar_a);
    pend_a = true;
  };
  auto issue_h = [&](int tile) {
    mbar_expect(bar_h, 2 * kAtom);
    tma_load_box(sb + kOffCat, &a.tm_h, 0, tile * 128, bar_h);
    tma_load_box(sb + kOffCat + kAtom, &a.tm_h, 64, tile * 128, bar_h);
    pend_h = true;
  };

  if (tid == 0 && first_tile < a.ntiles) {
    issue_a(first_tile);
    if (has_h) issue_h(first_tile);
    issue_weight(0);
    issue_weight(1);
  }

  bool stop = false;
  for (int it = 0; !stop && tile_of(it) < a.ntiles; it++) {
    const int tile = tile_of(it);
    const int row0 = tile * 128;
    const bool next = tile_of(it + 1) < a.ntiles;
    for (int li = 0; li < L && !stop; li++) {
      const Step st = step_of(a.mode, li);
      const Shape sh = layer_shape(a.mode, li);
      const int g = it * L + li;
      // producer: inputs and weight of this layer, then its MMAs
      if (tid == 0) {
        bool ok = true;
        if (li == 0) {
          ok = mbar_wait(bar_a, ph_a);
          ph_a ^= 1u;
          pend_a = false;
        }
        if (ok && li == 1 && has_h) {
          ok = mbar_wait(bar_h, ph_h);
          ph_h ^= 1u;
          pend_h = false;
        }
        if (ok) {
          ok = mbar_wait(bar_w[g & 1], ph_w[g & 1]);
          ph_w[g & 1] ^= 1u;
          pend_w[g & 1] = false;
        }
        if (ok) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          issue_mma(tmem, sb + st.a_off, sb + kOffW0 + (g & 1) * kSlotBytes, sh, sh.n == 256 ? id256 : id128, bar_m);
          pend_m = true;
        } else {
          fail_wait();
        }
      }
      __syncthreads();
      if (s_abort) break;
      // every thread: the accumulator of this layer
      bool ok = mbar_wait(bar_m, ph_m);
      ph_m ^= 1u;
      if (tid == 0) pend_m = false;
      if (!ok) fail_wait();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ok) {
        // the MMA has read its operands: refill the freed buffers
        if (tid == 0) {
          issue_weight(g + 2);
          if (next) {
            const bool a_free = (a.mode == CHAIN_ENCODER && li == 1) || (a.mode == CHAIN_ROUND && li == 2) ||
                                (a.mode == CHAIN_LAST && li == 4);
            const bool h_free = has_h && li == 3;
            if (a_free) issue_a(tile_of(it + 1));
            if (h_free) issue_h(tile_of(it + 1));
          }
        }
        if (st.epi == EPI_RESIDUAL && has_h) {
          if (!mbar_wait(bar_h, ph_h_all)) fail_wait();
          ph_h_all ^= 1u;
        }
        const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
        const int grow = row0 + r;
        const bool live = grow < a.n;
        const float *bias = a.layer[li].bias;
        const int ncol = st.epi == EPI_OUT ? 16 : sh.n;
        for (int c0 = 0; c0 < ncol; c0 += 16) {
          float v[16];
          tmem_ld16(taddr + c0, v);
          if (bias)
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] += bias[c0 + j];
          if (st.epi == EPI_RESIDUAL) {
            float h[16];
            smem_get16(sm + kOffCat, r, c0, h);
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] += h[j];
            smem_put16(sm + kOffCat, r, c0, v);
            if (live && a.h_out) global_put16(a.h_out + (size_t)grow * 128 + c0, v);
          } else if (st.epi == EPI_SMEM) {
            if (st.relu)
#pragma unroll
              for (int j = 0; j < 16; j++) v[j] = fmaxf(v[j], 0.0f);
            smem_put16(sm + st.dst, r, c0, v);
            if (st.h_global && live) global_put16(a.h_out + (size_t)grow * 128 + c0, v);
          } else if (st.epi == EPI_PQ) {
            if (live) global_put16(a.pq_out + (size_t)grow * 256 + c0, v);
          } else if (live) {
            float4 *dst = reinterpret_cast<float4 *>(a.out + (size_t)grow * 128 + c0);
#pragma unroll
            for (int j = 0; j < 4; j++) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          }
        }
      }
      // shared-memory results -> visible to the next layer's MMA (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (s_abort) stop = true;
    }
    if (s_abort) stop = true;
  }
  // after a failed wait: let every copy or MMA still in flight land first
  if (tid == 0) {
    if (pend_a) mbar_wait(bar_a, ph_a);
    if (pend_h) mbar_wait(bar_h, ph_h);
    for (int s = 0; s < 2; s++)
      if (pend_w[s]) mbar_wait(bar_w[s], ph_w[s]);
    if (pend_m) mbar_wait(bar_m, ph_m);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
}

__global__ void k_swizzle_image(const __nv_bfloat16 *__restrict__ W, int N, int K, uint8_t *__restrict__ img)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // one 16-byte chunk
  const int chunks = K / 8;
  if (i >= N * chunks) return;
  const int row = i / chunks, c = i % chunks;
  const int ka = c / 8, cc = c % 8;
  const uint4 v = *reinterpret_cast<const uint4 *>(W + (size_t)row * K + c * 8);
  *reinterpret_cast<uint4 *>(img + (size_t)ka * N * 128 + row * 128 + ((cc ^ (row & 7)) << 4)) = v;
}

}  // namespace

uph_status make_row_tensor_map(CUtensorMap *map, const void *base, int rows, int row_bytes)
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    const cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return fail(UPH_CUDA_ERROR, "cuTensorMapEncodeTiled is not available from the driver");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_bytes & 15) || rows < 1)
    return fail(UPH_BAD_ARG, "tensor map: base and row stride must be 16-byte aligned");
  cuuint64_t dims[2] = {128, static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(row_bytes)};
  cuuint32_t box[2] = {64, 128};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(UPH_CUDA_ERROR, "cuTensorMapEncodeTiled failed");
  return UPH_OK;
}

void launch_swizzle_image(const __nv_bfloat16 *W, int N, int K, uint8_t *img, cudaStream_t s)
{
  const int chunks = N * (K / 8);
  k_swizzle_image<<<(chunks + 255) / 256, 256, 0, s>>>(W, N, K, img);
}

uph_status launch_node_chain(const ChainArgs &a, cudaStream_t s)
{
  if (a.n < 1 || a.ntiles != (a.n + 127) / 128) return fail(UPH_BAD_ARG, "node chain: bad tile count");
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    UPH_CUDA(cudaGetDevice(&dev));
    UPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    UPH_CUDA(cudaFuncSetAttribute(k_node_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
  }
  const int grid = a.ntiles < sms ? a.ntiles : sms;
  k_node_chain<<<grid, kThreads, kSmemBytes, s>>>(a);
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

}  // namespace uph
