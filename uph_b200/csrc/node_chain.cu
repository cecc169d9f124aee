// Fused node-side layers of the surrogate network on the tcgen05 tensor cores.
//
// Between two edge layers every layer of the network is node-local, so a
// 128-row tile of nodes can run through all of them without leaving the SM:
//   encoder: F -> relu(E1 F + b) -> h0 = E2 (.) + b -> [P | Q] = W_pq h0 + b
//   round:   S, h -> m = W2 S -> u = relu(N1 [h ; m] + b) -> h' = h + N2 u + b
//            -> [P | Q]' = W_pq' h' + b        (or, in the last round,
//            -> relu(Dec1 h' + b) -> out = Dec2 (.) + b)
// Every weight is cut into 128 x 128 pieces (N1 into its two K halves, which
// accumulate into one TMEM tile; W_pq into its P and Q rows, which fill
// TMEM columns 0..127 and 128..255), each a K = 128, N = 128 UMMA.
//
// Two persistent CTAs per SM, 96 KiB of shared memory each:
//   X  2 atoms   the tile's first operand (F or S), then m, u, ... and P
//   H  2 atoms   h, updated in place by the residual layer
//   W  2 atoms   one weight piece (and Q while [P | Q] is stored)
// (an atom = 128 rows x 64 BF16 columns in the 128-byte-swizzled K-major
// layout of the UMMA descriptors).  Inputs arrive by TMA (2-D tensor maps
// with 128-byte swizzle, no multicast), weight pieces as pre-swizzled images
// by bulk copies, all completing on mbarriers.  One thread issues each
// piece's MMAs into the CTA's 256-column TMEM accumulator; after a layer's
// last piece the four warps read their 32 TMEM lanes (one row per thread),
// apply bias / residual / ReLU and write BF16 into shared memory; h and
// [P | Q] leave the SM as TMA tensor stores of those swizzled atoms.  One
// CTA's chain is serial (MMA -> epilogue -> next MMA); the other CTA on the
// SM fills its waits.
//
// The arithmetic is that of the unfused path (tc_gemm.cu) step for step --
// the same K order of MMAs, FP32 bias then residual, the same BF16 rounding
// points -- so both give the same network.
//
// Every mbarrier wait is bounded; a wait that gives up sets ERR_TIMEOUT, the
// CTA stops, waits (bounded) for its copies, stores and MMAs in flight, frees
// its TMEM and returns.
#include <cudaTypedefs.h>

#include <cute/arch/mma_sm100_desc.hpp>
#include <cute/numeric/numeric_types.hpp>

#include "node_chain.cuh"

namespace uph {
namespace {

constexpr int kAtom = 16384;           // 128 rows x 128 bytes
constexpr int kOffX = 0;               // 2 atoms: the tile's working activations
constexpr int kOffH = 2 * kAtom;       // 2 atoms: h
constexpr int kOffW = 4 * kAtom;       // 2 atoms: one weight piece (128 x 128)
constexpr int kSmemUsed = 6 * kAtom;   // 96 KiB: two CTAs per SM
constexpr int kSmemBytes = kSmemUsed + 1024;
constexpr int kThreads = 128;
constexpr int kPieceBytes = 2 * kAtom;
constexpr long long kWaitLimit = 1LL << 26;

enum Buf : int { BUF_X = 0, BUF_H = 1 };

// what the epilogue after a layer's last piece does with the accumulator
enum Epi : int {
  EPI_NONE = 0,      // not the layer's last piece
  EPI_X = 1,         // (+ bias) (ReLU) -> BF16 into X
  EPI_H = 2,         // + bias -> BF16 into H (the encoder's h0)
  EPI_RESIDUAL = 3,  // + bias + h -> BF16 into H
  EPI_PQ = 4,        // 256 columns + bias -> BF16, P staged in X and Q in the weight slot, stored by TMA
  EPI_OUT = 5,       // columns 0..15 + bias -> FP32 to out
};

struct PieceSpec {
  int a;     // A operand buffer
  int col;   // TMEM column of the accumulator
  int acc;   // accumulate onto it
  int epi;   // EPI_NONE for all but a layer's last piece
  int relu;
};

__host__ __device__ inline int piece_count(int mode) { return mode == CHAIN_ENCODER ? 4 : 6; }

// encoder: E1 | E2 | W_P W_Q;  round: W2 | N1a N1b | N2 | W_P W_Q;
// last round: W2 | N1a N1b | N2 | Dec1 | Dec2
__device__ __forceinline__ PieceSpec piece_of(int mode, int p)
{
  if (mode == CHAIN_ENCODER) {
    if (p == 0) return PieceSpec{BUF_X, 0, 0, EPI_X, 1};
    if (p == 1) return PieceSpec{BUF_X, 0, 0, EPI_H, 0};
    if (p == 2) return PieceSpec{BUF_H, 0, 0, EPI_NONE, 0};
    return PieceSpec{BUF_H, 128, 0, EPI_PQ, 0};
  }
  if (p == 0) return PieceSpec{BUF_X, 0, 0, EPI_X, 0};
  if (p == 1) return PieceSpec{BUF_H, 0, 0, EPI_NONE, 0};
  if (p == 2) return PieceSpec{BUF_X, 0, 1, EPI_X, 1};
  if (p == 3) return PieceSpec{BUF_X, 0, 0, EPI_RESIDUAL, 0};
  if (mode == CHAIN_ROUND) return p == 4 ? PieceSpec{BUF_H, 0, 0, EPI_NONE, 0} : PieceSpec{BUF_H, 128, 0, EPI_PQ, 0};
  return p == 4 ? PieceSpec{BUF_H, 0, 0, EPI_X, 1} : PieceSpec{BUF_X, 0, 0, EPI_OUT, 0};
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

// one 128-row x 64-column box from shared memory to a 2-D tensor map (x, y
// are non-negative and x * 2 bytes is a multiple of 16)
__device__ __forceinline__ void tma_store_box(const CUtensorMap *map, uint32_t src, int x, int y)
{
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(src), "r"(x), "r"(y)
               : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
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

// 64 consecutive TMEM columns of this warp's 32 lanes, waited for inside the
// same asm statement so no use of the registers can be scheduled before
// the load completes
__device__ __forceinline__ void tmem_ld64(uint32_t addr, float v[64])
{
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(addr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 64; j++) v[j] = __uint_as_float(r[j]);
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

// issue the K = 128 MMA of one 128 x 128 weight piece
__device__ __forceinline__ void issue_piece(uint32_t tmem, uint32_t a, uint32_t w, uint32_t idesc, int accumulate,
                                            uint32_t bar)
{
#pragma unroll
  for (int ka = 0; ka < 2; ka++)
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const uint64_t da = desc_sw128(a + ka * kAtom + kk * 32);
      const uint64_t db = desc_sw128(w + ka * kAtom + kk * 32);
      const uint32_t acc = (accumulate || ka || kk) ? 1u : 0u;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
          "l"(da), "l"(db), "r"(idesc), "r"(acc));
    }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__global__ void __launch_bounds__(kThreads, 2) k_node_chain(const __grid_constant__ ChainArgs a)
{
  extern __shared__ uint8_t smem_raw[];
  // X tile, h tile, weight piece, intermediate MMA, final MMA
  __shared__ uint64_t bars[5];
  __shared__ uint32_t tmem_slot;
  __shared__ int s_abort;
  __shared__ int s_mma_pending;  // set by the final drain: an MMA never completed
  __shared__ float s_bias[256];  // the current layer's bias
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = su32(sm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = warp * 32 + lane;  // tile row = TMEM lane of this thread
  const int NP = piece_count(a.mode);
  const bool has_h = a.mode != CHAIN_ENCODER;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_slot)), "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int b = 0; b < 5; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
    s_mma_pending = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t bar_x = su32(&bars[0]), bar_h = su32(&bars[1]), bar_w = su32(&bars[2]);
  const uint32_t bar_mi = su32(&bars[3]), bar_m = su32(&bars[4]);
  const uint32_t idesc = static_cast<uint32_t>(
      cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 128, cute::UMMA::Major::K,
                                  cute::UMMA::Major::K>());

  // barrier phases: every thread waits on bar_m (and on bar_h before the
  // residual); thread 0 also on the inputs, the weights and bar_mi
  uint32_t ph_m = 0, ph_h_all = 0, ph_x = 0, ph_h = 0, ph_w = 0, ph_mi = 0;
  bool pend_x = false, pend_h = false, pend_w = false, pend_mi = false, pend_m = false;
  const int stride = gridDim.x;
  const int first_tile = blockIdx.x;
  auto tile_of = [&](int it) { return first_tile + it * stride; };
  auto fail_wait = [&]() {
    s_abort = 1;
    atomicOr(a.err, ERR_TIMEOUT);
  };
  // thread 0; a wait that gave up leaves the phase pending, so the final
  // drain waits for that same phase again
  auto wait0 = [&](uint32_t bar, uint32_t &ph, bool &pend) {
    const bool ok = mbar_wait(bar, ph);
    if (ok) {
      ph ^= 1u;
      pend = false;
    }
    return ok;
  };
  // thread 0: piece g (piece g % NP of iteration g / NP) into the weight slot
  auto issue_weight = [&](int g) {
    if (tile_of(g / NP) >= a.ntiles) return;
    mbar_expect(bar_w, kPieceBytes);
    bulk_load(sb + kOffW, a.piece[g % NP].img, kAtom, bar_w);
    bulk_load(sb + kOffW + kAtom, a.piece[g % NP].img + kAtom, kAtom, bar_w);
    pend_w = true;
  };
  auto issue_x = [&](int tile) {
    mbar_expect(bar_x, 2 * kAtom);
    tma_load_box(sb + kOffX, &a.tm_a, 0, tile * 128, bar_x);
    tma_load_box(sb + kOffX + kAtom, &a.tm_a, 64, tile * 128, bar_x);
    pend_x = true;
  };
  auto issue_h = [&](int tile) {
    mbar_expect(bar_h, 2 * kAtom);
    tma_load_box(sb + kOffH, &a.tm_h, 0, tile * 128, bar_h);
    tma_load_box(sb + kOffH + kAtom, &a.tm_h, 64, tile * 128, bar_h);
    pend_h = true;
  };

  if (tid == 0 && first_tile < a.ntiles) {
    issue_weight(0);
    issue_x(first_tile);
    if (has_h) issue_h(first_tile);
  }

  bool stop = false;
  for (int it = 0; !stop && tile_of(it) < a.ntiles; it++) {
    const int row0 = tile_of(it) * 128;
    const bool next = tile_of(it + 1) < a.ntiles;
    for (int p = 0; p < NP && !stop; p++) {
      const PieceSpec ps = piece_of(a.mode, p);
      const int g = it * NP + p;
      // producer: weights (and this tile's inputs on first use), then the MMA
      if (tid == 0) {
        bool ok = wait0(bar_w, ph_w, pend_w);
        if (ok && p == 0) ok = wait0(bar_x, ph_x, pend_x);
        if (ok && p == 1 && has_h) ok = wait0(bar_h, ph_h, pend_h);
        if (ok) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          issue_piece(tmem + ps.col, sb + (ps.a == BUF_X ? kOffX : kOffH), sb + kOffW, idesc, ps.acc,
                      ps.epi == EPI_NONE ? bar_mi : bar_m);
          if (ps.epi == EPI_NONE) {
            pend_mi = true;
            // the next piece of this layer needs the slot: wait for the MMA
            ok = wait0(bar_mi, ph_mi, pend_mi);
            if (ok) issue_weight(g + 1);
          } else {
            pend_m = true;
          }
        }
        if (!ok) fail_wait();
      }
      if (ps.epi == EPI_NONE) continue;
      // the layer's bias to shared memory (the last epilogue is done)
      const float *bias = a.piece[p].bias;
      const int ncol = ps.epi == EPI_PQ ? 256 : ps.epi == EPI_OUT ? 16 : 128;
      if (bias)
        for (int c = tid; c < ncol; c += kThreads) s_bias[c] = bias[c];
      __syncthreads();
      if (s_abort) break;
      bool ok = mbar_wait(bar_m, ph_m);
      if (ok) {
        ph_m ^= 1u;
        if (tid == 0) pend_m = false;
      } else {
        fail_wait();
      }
      // Each thread polls on its own clock, so a wait can give up in some
      // threads only.  The warp-wide TMEM loads below need the whole warp;
      // s_abort, read after the next block barrier, stops every warp.
      ok = __all_sync(0xffffffffu, ok);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ok) {
        // the MMA has read its operands: refill what it freed
        if (tid == 0) {
          if (ps.epi != EPI_PQ) issue_weight(g + 1);  // after a [P | Q] layer the slot stages Q first
          if (next && a.mode == CHAIN_LAST) {
            if (p == 4) issue_h(tile_of(it + 1));
            if (p == 5) issue_x(tile_of(it + 1));
          }
        }
        if (ps.epi == EPI_RESIDUAL) {
          if (!mbar_wait(bar_h, ph_h_all)) fail_wait();
          ph_h_all ^= 1u;
        }
        const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
        if (ps.epi == EPI_OUT) {
          float v[16];
          tmem_ld16(taddr, v);
          const int grow = row0 + r;
#pragma unroll
          for (int j = 0; j < 16; j++) v[j] += s_bias[j];
          if (grow < a.n) {
            float4 *dst = reinterpret_cast<float4 *>(a.out + (size_t)grow * 128);
#pragma unroll
            for (int j = 0; j < 4; j++) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          }
        } else {
          for (int c64 = 0; c64 < ncol; c64 += 64) {
            float v[64];
            tmem_ld64(taddr + c64, v);
            if (bias)
#pragma unroll
              for (int j = 0; j < 64; j++) v[j] += s_bias[c64 + j];
#pragma unroll
            for (int q = 0; q < 4; q++) {
              float *w = v + 16 * q;
              const int c0 = c64 + 16 * q;
              if (ps.epi == EPI_RESIDUAL) {
                float h[16];
                smem_get16(sm + kOffH, r, c0, h);
#pragma unroll
                for (int j = 0; j < 16; j++) w[j] += h[j];
                smem_put16(sm + kOffH, r, c0, w);
              } else if (ps.epi == EPI_PQ) {
                if (c0 < 128)
                  smem_put16(sm + kOffX, r, c0, w);
                else
                  smem_put16(sm + kOffW, r, c0 - 128, w);
              } else {
                if (ps.relu)
#pragma unroll
                  for (int j = 0; j < 16; j++) w[j] = fmaxf(w[j], 0.0f);
                smem_put16(sm + (ps.epi == EPI_H ? kOffH : kOffX), r, c0, w);
              }
            }
          }
        }
      }
      // shared-memory results -> visible to the next MMA and the TMA stores
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (s_abort) {
        stop = true;
        continue;
      }
      const bool h_done = (ps.epi == EPI_RESIDUAL || ps.epi == EPI_H) && a.store_h;
      if (tid == 0 && (h_done || ps.epi == EPI_PQ)) {
        if (h_done) {
          tma_store_box(&a.tm_hout, sb + kOffH, 0, row0);
          tma_store_box(&a.tm_hout, sb + kOffH + kAtom, 64, row0);
        }
        if (ps.epi == EPI_PQ) {
          tma_store_box(&a.tm_pq, sb + kOffX, 0, row0);
          tma_store_box(&a.tm_pq, sb + kOffX + kAtom, 64, row0);
          tma_store_box(&a.tm_pq, sb + kOffW, 128, row0);
          tma_store_box(&a.tm_pq, sb + kOffW + kAtom, 192, row0);
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        if (ps.epi == EPI_PQ) {
          // the stores have read X, h and the slot: refill them
          asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          issue_weight(g + 1);
          if (next) {
            issue_x(tile_of(it + 1));
            if (has_h) issue_h(tile_of(it + 1));
          }
        }
      }
      if (ps.epi == EPI_PQ) __syncthreads();
    }
  }
  // normal end or a failed wait: let every copy, store or MMA in flight land
  // (bounded again).  An MMA that still has not completed may write the
  // accumulator: its TMEM is then left allocated rather than freed under it.
  if (tid == 0) {
    bool mma_done = true;
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    if (pend_x) mbar_wait(bar_x, ph_x);
    if (pend_h) mbar_wait(bar_h, ph_h);
    if (pend_w) mbar_wait(bar_w, ph_w);
    if (pend_mi && !mbar_wait(bar_mi, ph_mi)) mma_done = false;
    if (pend_m && !mbar_wait(bar_m, ph_m)) mma_done = false;
    if (!mma_done) {
      fail_wait();
      s_mma_pending = 1;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0 && !s_mma_pending)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
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

uph_status make_row_tensor_map(CUtensorMap *map, const void *base, int rows, int cols, int row_bytes)
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
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_bytes & 15) || rows < 1 || cols % 64)
    return fail(UPH_BAD_ARG, "tensor map: base and row stride must be 16-byte aligned, columns whole boxes");
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
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
  for (int p = 0; p < (a.mode == CHAIN_ENCODER ? 4 : 6); p++)
    if (!a.piece[p].img || (reinterpret_cast<uintptr_t>(a.piece[p].img) & 15))
      return fail(UPH_BAD_ARG, "node chain: missing or misaligned weight piece");
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    UPH_CUDA(cudaGetDevice(&dev));
    UPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    UPH_CUDA(cudaFuncSetAttribute(k_node_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
  }
  const int grid = a.ntiles < 2 * sms ? a.ntiles : 2 * sms;
  k_node_chain<<<grid, kThreads, kSmemBytes, s>>>(a);
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

}  // namespace uph
