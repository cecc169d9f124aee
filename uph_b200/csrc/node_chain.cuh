// Fused node-side layers of the surrogate network (node_chain.cu).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "uph_internal.cuh"

namespace uph {

// One 128 x 128 weight piece of a chain as a pre-swizzled shared-memory
// image (2 atoms of 128 rows x 128 bytes, 16-byte chunk c of row r at
// r * 128 + ((c ^ (r % 8)) * 16)) and, on a layer's last piece, the layer's
// FP32 bias (256 values after the two [P | Q] pieces), else null.
struct ChainPiece {
  const uint8_t *img;
  const float *bias;
};

enum ChainMode : int {
  CHAIN_ENCODER = 0,  // F -> relu(E1) -> E2 = h0 -> PQ0
  CHAIN_ROUND = 1,    // S, h -> m = W2 S -> u = relu(N1 [h ; m]) -> h' = h + N2 u -> PQ'
  CHAIN_LAST = 2,     // S, h -> m -> u -> h' -> relu(Dec1 h') -> out = Dec2 (.)
};

struct ChainArgs {
  CUtensorMap tm_a;     // the first operand's rows: F (encoder) or S [n x 128] BF16
  CUtensorMap tm_h;     // h [n x 128] BF16 (rounds)
  CUtensorMap tm_hout;  // h' [n x 128] BF16 (store_h)
  CUtensorMap tm_pq;    // [P | Q]' [n x 256] BF16 (encoder, rounds but the last)
  int mode;
  int n, ntiles;
  int store_h;
  ChainPiece piece[6];  // encoder: E1 E2 W_P W_Q; rounds: W2 N1a N1b N2 (W_P W_Q | Dec1 Dec2)
  float *out;           // [n x 128]; the last round writes columns 0..15
  unsigned *err;
};

// 2-D BF16 tensor map over a row-major [rows x cols] matrix with row stride
// `row_bytes`, boxes of 128 rows x 64 columns, 128-byte swizzle (loads and
// stores of one shared-memory atom).
uph_status make_row_tensor_map(CUtensorMap *map, const void *base, int rows, int cols, int row_bytes);
// writes the shared-memory image of W [N x K] (row-major BF16) to img: K/64
// atoms of N rows x 128 bytes
void launch_swizzle_image(const __nv_bfloat16 *W, int N, int K, uint8_t *img, cudaStream_t s);
uph_status launch_node_chain(const ChainArgs &a, cudaStream_t s);

}  // namespace uph
