// Device-resident schedule of the batched H-matrix-vector product (built on the host by
// the engine from the leaf list, consumed by gemv.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hmatb200 {

struct GemvFullLeaf {
  int row_off, m, col_off, n;
  long long off;  // element offset in the full arena (column-major m x n)
};

struct GemvRkLeaf {
  int row_off, m, col_off, n, k, pad;
  long long off;   // element offset of A (m x k), B (n x k) follows
  long long zoff;  // element offset of this leaf's z (k x 16 slots) in the z buffer
};

// A chunk [start, start + len) of the rows of B ('N') or A ('T') of one Rk leaf.
struct GemvZItem {
  int leaf, start, len, pad;
  long long dst_off;  // where its k x R partial goes in the z buffer
};

// One output block: rows [off, off + len) of y in cluster order, fed by `count` entries.
struct GemvYBlock {
  int off, len, first, count;
};
struct GemvYEntry {
  int type;  // 0 full leaf, 1 rk leaf
  int leaf;  // index in the full or rk table
  int sub;   // offset of the block inside the leaf's rows ('N') or cols ('T')
  int pad;
};

struct GemvSide {
  int nzitems = 0;
  const GemvZItem* zitems = nullptr;
  int nmulti = 0;  // leaves split into several items
  const int* multi = nullptr;
  const int* mfirst = nullptr;
  const int* mcount = nullptr;
  int nblocks = 0;
  const GemvYBlock* blocks = nullptr;
  const GemvYEntry* entries = nullptr;
  int GS = 64;  // threads per row group in the y-phase
};

// Optional per-phase timing of one eager product: events recorded before the gather and
// after the gather, z-phase (+ reduction) and y-phase.
struct GemvTiming {
  cudaEvent_t ev[4];
};

struct GemvPlan {
  int n_rows = 0, n_cols = 0;
  const int* perm_rows = nullptr;  // internal -> client, rows
  const int* perm_cols = nullptr;
  int nfull = 0, nrk = 0;
  const GemvFullLeaf* full = nullptr;
  const GemvRkLeaf* rk = nullptr;
  const void* full_arena = nullptr;
  const void* rk_arena = nullptr;
  GemvSide side_n, side_t;
  long long z_elems = 0;
};

}  // namespace hmatb200
