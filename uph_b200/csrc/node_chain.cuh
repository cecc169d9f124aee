// Fused node-side layers of the surrogate network (node_chain.cu).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "uph_internal.cuh"

namespace uph {

// One layer of a chain: its weight matrix as a pre-swizzled shared-memory
// image (K/64 atoms of N rows x 128 bytes, 16-byte chunk c of row r at
// r * 128 + ((c ^ (r % 8)) * 16)) and its FP32 bias (or null).
struct ChainLayer {
  const uint8_t *img;
  const float *bias;
};

enum ChainMode : int {
  CHAIN_ENCODER = 0,  // F -> relu(E1) -> E2 = h0 -> PQ0
  CHAIN_ROUND = 1,    // S, h -> m = W2 S -> u = relu(N1 [h ; m]) -> h' = h + N2 u -> PQ'
  CHAIN_LAST = 2,     // S, h -> m -> u -> h' -> relu(Dec1 h') -> out = Dec2 (.)
};

struct ChainArgs {
  CUtensorMap tm_a;   // the first operand's rows: F (encoder) or S [n x 128] BF16
  CUtensorMap tm_h;   // h [n x 128] BF16 (rounds)
  int mode;
  int n, ntiles;
  ChainLayer layer[5];
  __nv_bfloat16 *h_out;  // [n x 128]
  __nv_bfloat16 *pq_out; // [n x 256]
  float *out;            // [n x 128]; the last round writes columns 0..15
  unsigned *err;
};

// 2-D BF16 tensor map over a row-major [rows x 128] matrix with row stride
// `row_bytes`, boxes of 128 rows x 64 columns, 128-byte swizzle.
uph_status make_row_tensor_map(CUtensorMap *map, const void *base, int rows, int row_bytes);
// writes the shared-memory image of W [N x K] (row-major BF16) to img
void launch_swizzle_image(const __nv_bfloat16 *W, int N, int K, uint8_t *img, cudaStream_t s);
uph_status launch_node_chain(const ChainArgs &a, cudaStream_t s);

}  // namespace uph
