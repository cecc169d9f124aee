// Tiled execution of a rate pass: one CTA per storage tile of T x T cells.
//
// The CTA stages every particle of its tile and of the `reach` cells around
// it (the "block") into shared memory as one record each, then lets each
// thread own one fluid particle of the tile's core cells and walk its
// neighbour stencil inside the block.  A record is read from global memory
// once per CTA instead of once per neighbour (about 20 times), and the pair
// loop reads partners with a few 16-byte shared-memory loads.
//
// Order: the block's records are the cell list's row ranges, row by row, so
// a stencil row is one contiguous range of records, and partners are visited
// in exactly the cell list's order (rows bottom to top, cells left to right,
// each cell's slots ascending) -- the order of the global walk.  A CTA whose
// block holds more records than fit (a crowded tile) walks the cell list in
// global memory instead, with the same arithmetic and the same order, so
// either way every particle's sums are the same.
#pragma once

#include <algorithm>

#include "pass_common.cuh"

namespace uph {

constexpr int kTileThreads = 256;  // threads of a tiled pass CTA
constexpr int kTileChunk = 24;     // partners listed per thread before they are processed
constexpr int kTileRowsMax = 32;   // rows and columns of a block (tile + 2 reach)
constexpr int kTileTabMax = (kTileRowsMax + 1) * kTileRowsMax;
constexpr unsigned short kRoleI16 = 0x8000u;  // list-entry flag: this particle is the pair's i

// one CTA's tile and block, in shared memory
// a global line fetched into L2 ahead of its use
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

struct TileBlock {
  int bx0, by0, W, H;          // block: first cell (x, y) and size in cells
  int ncore;                   // particles (of any kind) in the core cells
  int nrec;                    // particles in the block
  int gs[kTileRowsMax];        // cell-list position of each block row's first particle
  int roff[kTileRowsMax + 1];  // record index of each block row's first particle
  int cs0[kTileRowsMax];       // cell-list position of each core row's first particle
  int coff[kTileRowsMax + 1];  // index among the core's particles of each row's first
  int tab[kTileTabMax];        // record index of block cell (r, c): tab[r (W + 1) + c]
};

// Fills B for tile `tile_id` (all threads; ends with a barrier).  One round
// of global loads: the cell-list start of every block cell and of the cell
// after each block row (which also give the core rows' ranges, the tile's
// columns lying inside the block), kept in tab; the row scans and the
// record indices then come from shared memory.
__device__ __forceinline__ void tile_setup(const DevParams &P, const CellGrid &G, int tile_id, TileBlock &B)
{
  const int T = P.tile, R = P.reach;
  const int tx = tile_id % P.ntx, ty = tile_id / P.ntx;
  const int cx0 = tx * T, cy0 = ty * T;
  const int bx0 = max(cx0 - R, 0), bx1 = min(cx0 + T - 1 + R, P.ncx - 1);
  const int by0 = max(cy0 - R, 0), by1 = min(cy0 + T - 1 + R, P.ncy - 1);
  const int W = bx1 - bx0 + 1, H = by1 - by0 + 1;
  for (int e = threadIdx.x; e < (W + 1) * H; e += blockDim.x) {
    const int r = e / (W + 1), c = e % (W + 1);
    B.tab[e] = G.start[(by0 + r) * P.ncx + bx0 + c];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int r = threadIdx.x;
    int len = 0, clen = 0, gsr = 0, cs0r = 0;
    if (r < H) {
      const int *row = B.tab + r * (W + 1);
      gsr = row[0];
      len = row[W] - gsr;
      const int cr = by0 + r - cy0;
      if (cr >= 0 && cr < T) {
        // the tile's columns cx0 .. cx0 + T - 1 lie inside the block (ncx is
        // a multiple of T), so their starts and the one after are in tab
        cs0r = row[cx0 - bx0];
        clen = row[cx0 + T - bx0] - cs0r;
      }
    }
    int il = len, ic = clen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int a = __shfl_up_sync(0xffffffffu, il, o);
      const int c = __shfl_up_sync(0xffffffffu, ic, o);
      if (r >= o) {
        il += a;
        ic += c;
      }
    }
    B.gs[r] = gsr;
    B.roff[r] = il - len;
    B.cs0[r] = cs0r;
    B.coff[r] = ic - clen;
    if (r == 31) {
      B.roff[32] = il;
      B.coff[32] = ic;
      B.nrec = il;
      B.ncore = ic;
      B.bx0 = bx0;
      B.by0 = by0;
      B.W = W;
      B.H = H;
    }
  }
  __syncthreads();
  // list positions -> record indices of the block
  for (int e = threadIdx.x; e < (W + 1) * H; e += blockDim.x) {
    const int r = e / (W + 1);
    B.tab[e] = B.roff[r] + (B.tab[e] - B.gs[r]);
  }
  __syncthreads();
}

// the largest r with off[r] <= k, for k in [0, off[32])
__device__ __forceinline__ int tile_row_of(const int *off, int k)
{
  int r = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (off[r + step] <= k) r += step;
  return r;
}

// record index and cell-list position of the k-th particle of the core
__device__ __forceinline__ void tile_core(const TileBlock &B, int k, int &rec, int &pos)
{
  const int r = tile_row_of(B.coff, k);
  pos = B.cs0[r] + (k - B.coff[r]);
  const int br = r;  // core rows are block rows with the same index
  rec = B.roff[br] + (pos - B.gs[br]);
}

// The same, with the grid cell (cx, cy) the particle is listed in: the
// block cell of its row whose record range holds rec (the largest column
// whose first record is <= rec), from tab, without a global load.
__device__ __forceinline__ void tile_core_cell(const TileBlock &B, int k, int &rec, int &pos, int &cx, int &cy)
{
  const int r = tile_row_of(B.coff, k);
  pos = B.cs0[r] + (k - B.coff[r]);
  rec = B.roff[r] + (pos - B.gs[r]);
  const int *row = B.tab + r * (B.W + 1);
  int c = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (c + step < B.W && row[c + step] <= rec) c += step;
  cx = B.bx0 + c;
  cy = B.by0 + r;
}

// cell-list position of record k of the block
__device__ __forceinline__ int tile_record_pos(const TileBlock &B, int k)
{
  const int r = tile_row_of(B.roff, k);
  return B.gs[r] + (k - B.roff[r]);
}

// Walks a particle's stencil inside the block: (2 reach + 1) rows of
// (2 reach + 1) cells, each row one range of record indices.
struct BlockCursor {
  int row, row1, c0, c1, k, kend, stride;
  const int *tab;

  __device__ __forceinline__ void init(const TileBlock &B, int reach, int cx, int cy)
  {
    const int lc = cx - B.bx0, lr = cy - B.by0;
    c0 = max(lc - reach, 0);
    c1 = min(lc + reach, B.W - 1);
    row = max(lr - reach, 0);
    row1 = min(lr + reach, B.H - 1);
    stride = B.W + 1;
    tab = B.tab;
    k = tab[row * stride + c0];
    kend = tab[row * stride + c1 + 1];
  }
  __device__ __forceinline__ bool advance()
  {
    while (k >= kend) {
      if (++row > row1) return false;
      k = tab[row * stride + c0];
      kend = tab[row * stride + c1 + 1];
    }
    return true;
  }
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

// The cell list's walk as a source of slots (the global fallback).
struct GlobalCursor {
  NeighbourCursor c;
  const int *list;
  template <int kBatch>
  __device__ __forceinline__ int next_batch(int &pos) { return c.next_batch<kBatch>(pos); }
  __device__ __forceinline__ int at(int pos) const { return list[pos]; }
};
struct StagedCursor {
  BlockCursor c;
  template <int kBatch>
  __device__ __forceinline__ int next_batch(int &pos) { return c.next_batch<kBatch>(pos); }
  __device__ __forceinline__ int at(int pos) const { return pos; }
};

// The single-precision pre-test of phase 1: positions relative to the CTA's
// block origin in FP32 (exact enough to decide every candidate whose r^2 is
// not within a relative `band` of the cut-off), the exact FP64 test only
// for the rest.  `band` bounds the FP32 error of r^2 relative to the cut-off
// with a wide margin: the block spans E = max(W, H) cells, so each relative
// coordinate carries at most E cell 2^-24 of rounding and r^2 at most
// 4 R E cell 2^-24 + R^2 2^-23; band = 32 (E cell / R) 2^-23 + 2^-20.
struct F32Test {
  float xa, ya;  // own position relative to the origin
  float lo, hi;  // r2cut (1 -+ band): surely inside below lo, surely outside above hi
  float tiny;    // below this, r^2 may be at the DBL_EPSILON coincidence test: exact
  float vl;      // the candidate lists' radius squared (1 + band)
};

__device__ __forceinline__ F32Test make_f32_test(const DevParams &P, const TileBlock &B, float xa, float ya)
{
  const double R = sqrt(P.r2cut);
  const double E = (double)max(B.W, B.H) * P.cell;
  const double band = 32.0 * (E / R) * 0x1p-23 + 0x1p-20;
  // between two builds a particle moves at most the skin along each axis,
  // so a pair's distance shrinks by at most 2 sqrt(2) skin
  const double Rl = R + 2.0 * 1.4142135623730951 * P.skin;
  return F32Test{xa, ya, (float)(P.r2cut * (1.0 - band)), (float)(P.r2cut * (1.0 + band)),
                 (float)(P.r2cut * 1e-3), (float)(Rl * Rl * (1.0 + band))};
}

// The own particle's (slot a) candidate list for its listing.  use (the
// tile's lists are current) and no overflow: the entries are copied into
// column col of s_nb and their count returned.  Else -1: the stencil is
// walked, and vl_out points at the particle's list to write meanwhile (null
// when the lists are current but this one overflowed).
static_assert(kVlMax == 24 && kVlMax <= kTileChunk, "a candidate list is three 16-byte words and fits a column");
__device__ __forceinline__ int load_candidates(const CellGrid &G, int a, bool use, unsigned short *s_nb, int col,
                                               unsigned short *&vl_out)
{
  vl_out = nullptr;
  if (!use) {
    vl_out = G.vl + (size_t)a * kVlMax;
    return -1;
  }
  const uint4 *w = reinterpret_cast<const uint4 *>(G.vl + (size_t)a * kVlMax);
  const uint4 w0 = w[0], w1 = w[1], w2 = w[2];
  const int n = G.vl_n[a];
  if (n == kVlOverflow) return -1;
  const unsigned v[12] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
#pragma unroll
  for (int q = 0; q < 12; q++) {
    if (2 * q < n) s_nb[(2 * q) * kTileThreads + col] = (unsigned short)(v[q] & 0xffffu);
    if (2 * q + 1 < n) s_nb[(2 * q + 1) * kTileThreads + col] = (unsigned short)(v[q] >> 16);
  }
  return n;
}

// One batch of kB candidates b[] (the own index `self` for none) of the
// listing: the FP32 pre-test (kF32), the exact predicate and the pair
// filters; each listed partner goes to row cnt of column col of s_nb.
// vl_out (may be null): candidates within the list radius are appended to
// the own particle's candidate list, vl_cnt counting them past kVlMax too.
template <bool kBrute, bool kKnn, bool kF32, int kB, typename Src, typename Entry>
__device__ __forceinline__ void list_batch(const DevParams &P, const Src &src, int (&b)[kB], int self, int oa,
                                           double xa, double ya, const F32Test &ft, Entry *s_nb, int col, int &cnt,
                                           unsigned &my_pairs, int &my_nb, double &bx, double &by, double cd, int cj,
                                           unsigned short *vl_out, int &vl_cnt)
{
  constexpr Entry kRole = sizeof(Entry) == 2 ? (Entry)kRoleI16 : (Entry)kRoleI;
  bool sure[kB];  // FP32 says: surely inside and not coincident
  if constexpr (kF32) {
    float2 f[kB];
#pragma unroll
    for (int u = 0; u < kB; u++) f[u] = src.xyf(b[u]);
#pragma unroll
    for (int u = 0; u < kB; u++) {
      const float dxf = ft.xa - f[u].x, dyf = ft.ya - f[u].y;
      const float r2f = fmaf(dxf, dxf, dyf * dyf);
      if (vl_out && b[u] != self && r2f < ft.vl) {
        if (vl_cnt < kVlMax) vl_out[vl_cnt] = (unsigned short)b[u];
        vl_cnt++;
      }
      if (r2f > ft.hi) b[u] = self;  // surely outside: drop
      sure[u] = r2f < ft.lo && r2f > ft.tiny;
    }
  } else {
#pragma unroll
    for (int u = 0; u < kB; u++) sure[u] = false;
  }
#pragma unroll
  for (int u = 0; u < kB; u++) {
    if (b[u] == self) continue;
    double r2 = 0.0, dxa = 0.0, dya = 0.0;
    const bool exact = !sure[u] || kBrute || kKnn;
    if (exact) {
      const double2 q = src.xy(b[u]);
      dxa = xa - q.x;
      dya = ya - q.y;
      r2 = exact_r2(dxa, dya);
      if (!(r2 < P.r2cut)) continue;
    }
    const int ob = src.orig(b[u]);
    if (kBrute && ob >= P.b0 && ob < P.b1) brute_wall_force(P, r2, dxa, dya, src.mass(b[u]), bx, by);
    if (exact && r2 <= DBL_EPSILON) continue;
    my_nb++;
    if (max(oa, ob) >= P.pb) continue;
    const bool isI = ob > oa;
    if constexpr (kKnn) {
      double pd;
      int pj;
      if (!isI) src.cut(b[u], pd, pj);
      if (!(isI ? knn_key_le(r2, ob, cd, cj) : knn_key_le(r2, oa, pd, pj))) continue;
    }
    my_pairs += isI;
    s_nb[cnt++ * kTileThreads + col] = (Entry)b[u] | (isI ? kRole : (Entry)0);
  }
}

// Phase 1 of a rate pass: lists up to kChunk in-radius partners of the own
// particle (index `self` in the source) into column `col` of s_nb (row
// stride kTileThreads), four candidates at a time, each entry the partner's
// index with the role flag set when the own particle is the pair's i.  A
// partner is in-radius and in the reference's pair list exactly as in
// list_partners (pass_common.cuh): the decision is always the exact FP64
// predicate; with kF32 the FP32 pre-test (F32Test) settles the candidates
// far from the cut-off and the FP64 r^2 is computed only near it.  The
// brute-force wall modes see every in-radius boundary candidate.  The source
// gives xy(k), xyf(k) (kF32), orig(k), mass(k).
// kKnn: the reference's k-nearest cap (DevParams::knn): a pair is kept iff
// the partner is among query i's kept points -- the own particle's cut
// (cd, cj) when it is i, the partner's (src.cut(b)) when the partner is i.
// vl_out, vl_cnt: the candidate list written meanwhile (list_batch).
template <bool kBrute, int kChunk, bool kKnn, bool kF32, typename Src, typename Cursor, typename Entry>
__device__ __forceinline__ int tile_list(const DevParams &P, const Src &src, Cursor &cur, bool &more, int self,
                                        int oa, double xa, double ya, const F32Test &ft, Entry *s_nb, int col,
                                        unsigned &my_pairs, int &my_nb, double &bx, double &by, double cd, int cj,
                                        unsigned short *vl_out, int &vl_cnt)
{
  constexpr int kB = 4;
  int cnt = 0;
  while (more && cnt <= kChunk - kB) {
    int pos;
    const int n = cur.template next_batch<kB>(pos);
    if (n == 0) {
      more = false;
      break;
    }
    int b[kB];
#pragma unroll
    for (int u = 0; u < kB; u++) b[u] = (u < n) ? cur.at(pos + u) : self;
    list_batch<kBrute, kKnn, kF32, kB>(P, src, b, self, oa, xa, ya, ft, s_nb, col, cnt, my_pairs, my_nb, bx, by, cd,
                                       cj, vl_out, vl_cnt);
  }
  return cnt;
}

// The listing from the own particle's candidate list, which the caller has
// copied into rows 0 .. nshort - 1 of column col of s_nb: filtered in place
// (a listed partner is written at a row not above the one it was read
// from), in the list's order, which is the stencil walk's.  nshort <=
// kVlMax <= the rows of s_nb.
template <bool kBrute, bool kKnn, typename Src, typename Entry>
__device__ __forceinline__ int tile_list_short(const DevParams &P, const Src &src, int nshort, int self, int oa,
                                              double xa, double ya, const F32Test &ft, Entry *s_nb, int col,
                                              unsigned &my_pairs, int &my_nb, double &bx, double &by, double cd,
                                              int cj)
{
  constexpr int kB = 4;
  int cnt = 0, none = 0;
  for (int j = 0; j < nshort; j += kB) {
    int b[kB];
#pragma unroll
    for (int u = 0; u < kB; u++) b[u] = (j + u < nshort) ? (int)s_nb[(j + u) * kTileThreads + col] : self;
    list_batch<kBrute, kKnn, true, kB>(P, src, b, self, oa, xa, ya, ft, s_nb, col, cnt, my_pairs, my_nb, bx, by, cd,
                                       cj, nullptr, none);
  }
  return cnt;
}

// A pass CTA's statistics: warp reductions, then one atomic per warp into
// the counters the cell-list launch zeroed.
__device__ __forceinline__ void pass_stats(const PassStats &st, unsigned my_pairs, int my_nb)
{
  const unsigned wp = __reduce_add_sync(0xffffffffu, my_pairs);
  const int wn = (int)__reduce_max_sync(0xffffffffu, (unsigned)my_nb);
  if ((threadIdx.x & 31) == 0) {
    if (wp) atomicAdd(st.niac, (unsigned long long)wp);
    if (wn) atomicMax(st.max_nb, wn);
  }
}

}  // namespace uph
