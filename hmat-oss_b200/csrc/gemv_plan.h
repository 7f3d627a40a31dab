// Device-resident schedule of the batched H-matrix-vector product (built on the host by
// the engine from the leaf list, consumed by gemv.cu).
//
// Leaf storage is panelised so that every product term is one contiguous chunk:
//  * a full leaf F (m x n) is stored as row panels, one per output block of its rows,
//    each panel column-major (len x n);
//  * an Rk leaf stores A as row panels (len x k, column-major) and B transposed,
//    B^T column-major (k x n), i.e. each row of B contiguous.
// An output block is a leaf of the output cluster tree, cut into pieces of at most 128 rows.
//
// A product is a list of tasks; a task is one output (an output block of y, or the z = B^T x
// slot of an Rk leaf) accumulated from a list of units; a unit is out += op(P) X for one
// contiguous piece P of the leaf arena and one contiguous piece X of the xz buffer (x in
// cluster order, row-major, followed by the z rows).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hmatb200 {

// X rows of a unit come from at most kUnitRuns runs of consecutive xz rows (the columns of a
// block's matrix belong to several leaves, whose x or z rows are not adjacent).
constexpr int kUnitRuns = 4;

struct GemvUnit {
  long long poff;  // element offset of the piece P in the arena (16-byte aligned)
  int xrow;        // first row of the X piece in the xz buffer (nruns == 0)
  int c;           // inner extent (rows of X)
  int o0, ow;      // transposed units: output rows [o0, o0 + ow) this piece covers;
                   // other units: o0 = byte offset of the X rows in a warp-level pipeline
                   // stage (the piece's capacity; the FP32 tensor-core kernel reads it per unit)
  int pel;         // elements of the piece P (O x c, or c x ow when transposed)
  int shift;       // elements between the 16-byte aligned copy start and the piece
  int nruns;       // 0: X rows xrow .. xrow + c - 1; else X rows from the runs below, in order
  int run_row[kUnitRuns];
  unsigned short run_len[kUnitRuns];
};

struct GemvTask {
  int O;           // output rows
  int first_unit;  // units [first_unit, first_unit + nunits) in order
  int nunits;
  int out_row;     // y: first output row (cluster order); z: first xz row of the slot
  int red = -1;    // 'N' z chunk of a long group: its z sum (GemvZred index); the last chunk of
                   // the sum to finish adds the partial slots in part order
};

// One launch: tasks of one shape class, each CTA of a persistent grid takes a contiguous
// range [cta_begin[b], cta_begin[b + 1]) of tasks.
struct GemvLaunch {
  int ntasks = 0;
  int ncta = 0;
  const GemvTask* tasks = nullptr;
  const int* cta_begin = nullptr;  // warp-level launches: one range per warp (ncta * 4 + 1 entries)
  int rpt = 1;          // rows per lane: output rows <= 32 * rpt
  int ol = 32;          // output lanes (16 or 32)
  bool transposed = false;
  bool out_is_y = false;
  // Warp-level launches ('N' products): each warp owns whole tasks and pipelines its own
  // units.  map 3 (FP32): tensor-core tiles, at most 16 * rpt rows; map 2: column-slice
  // window over tasks of at most 32 rows (rpt rows per lane); map 1: half-warp row groups
  // (at most 64 rows); map 0: lanes over rows (at most 128).
  bool warp_level = false;
  // map 4 (FP32 'N' y launches, not warp-level): the tensor-memory kernel, one task at a time
  // per CTA, units of at most kTcCols columns and kTcPieceBytes bytes; it writes partial rows
  // like the warp-level launches.
  int map = 0;
};

// The arena's y region: per output block, the row panels of every leaf covering it side by side
// (full leaves n columns, Rk leaves their A panel of k columns) as one column-major matrix
// whose width is a multiple of kYColAlign (zero columns at the end, their X rows the zero rows
// of the xz buffer, kZeroRows of them after the x part).
constexpr int kYColAlign = 8;
constexpr int kZeroRows = 8;

// Unit capacities of the tensor-memory kernel: columns, piece bytes (128 rows x kTcCols),
// X rows bytes (kTcCols rows of 16 floats).
constexpr int kTcCols = 32;
constexpr int kTcPieceBytes = 128 * kTcCols * 4;
constexpr int kTcXBytes = kTcCols * 16 * 4;

// Per-stage capacities of the warp-level pipeline (bytes): one P piece and its X rows.  FP32
// pieces are 5,088 B: four CTAs of the tensor-core kernel (4 warps, two stages of 5,088 +
// 2,048 B a warp, 57.2 KB a CTA, 1 KB reserved) fill an SM's 228 KB, and the kernel's output
// tiles get the registers of four CTAs.  Against 3,584-B pieces at five CTAs an SM for the
// z-phase (the y-phase's 6 to 8 tiles already ran at four), fewer and larger units took the
// y-phase of the 100,000-point cylinder from 0.148 to 0.132 ms with the z-phase unchanged: per
// unit the kernel pays its barrier wait, descriptor and copy issue, and the larger pieces also
// keep more bytes in flight a warp.
// The FP64 and complex kernels use the same stage (the FP64 y-phase: 0.420 -> 0.403 ms against
// 4,096-byte pieces).
__host__ __device__ constexpr int warp_piece_bytes(int /*elem_bytes*/) { return 5088; }
constexpr int kWarpXBytes = 2048;
// FP32 units of short pieces (the z-phase's k x c blocks of B^T) may split the same stage the
// other way, kWarpXBytesWide bytes of X rows after a piece of the rest.
constexpr int kWarpXBytesWide = 3584;

// A long leaf whose z is computed in several chunks: the chunks' partial slots
// (nparts consecutive slots of k rows from part_row) are summed into final_row.
struct GemvZred {
  int final_row, k, part_row, nparts;
};

struct GemvSide {
  static const int kMaxLaunch = 8;
  int nz = 0;  // z-phase launches (one per rank class)
  GemvLaunch z[kMaxLaunch];
  int nzred = 0;
  const GemvZred* zred = nullptr;
  // zfused: the z kernels sum the parts themselves (the 'N' side); zcnt[i]: chunks of sum i
  // finished in the current product (cleared by the gather that opens every product)
  bool zfused = false;
  int* zcnt = nullptr;
  GemvLaunch y;
  const GemvUnit* units = nullptr;
  // The y launches write partial rows (chunks of the output blocks) into xz; the final pass
  // reads, per client row i, yrows[i] = {xz row of part 0, nparts << 8 | O}.
  int nyrows = 0;
  const int2* yrows = nullptr;
};

struct GemvFullLeaf {
  int row_off, m, col_off, n;
  long long goff;  // canonical offset (gradients, payload): column-major m x n
};
struct GemvRkLeaf {
  int row_off, m, col_off, n, k, pad;
  long long goff;   // canonical offset: A (m x k) then B (n x k), column-major
  int zrow_n, zrow_t;  // xz rows of z = B^T x ('N') and z' = A^T x ('T' / 'C')
};

// Status block of the products of one matrix, in device memory.  A kernel whose bounded
// wait for a bulk copy gives up sets `failed` (after waiting, again bounded, for the copies
// it has in flight) and stops; the host reads and clears it.  `wait_limit` bounds each wait
// (polls of a stage barrier); the drain after a give-up uses kGemvDrainLimit.
struct GemvStatus {
  int failed;
  int pad;
  long long wait_limit;
};
constexpr long long kGemvWaitLimit = 1LL << 26;
constexpr long long kGemvDrainLimit = 1LL << 26;

struct GemvTiming {
  cudaEvent_t ev[4];
};

struct GemvPlan {
  int n_rows = 0, n_cols = 0;
  int n_in_max = 0;      // rows of the x part of the xz buffer (kZeroRows zero rows follow it)
  long long xz_rows = 0; // total rows of the xz buffer (x part, zero rows, z slots, partial slots)
  const int* perm_rows = nullptr;  // internal -> client
  const int* perm_cols = nullptr;
  const int* iperm_rows = nullptr;  // client -> internal
  const int* iperm_cols = nullptr;
  const void* arena = nullptr;
  int nfull = 0, nrk = 0;
  const GemvFullLeaf* full = nullptr;
  const GemvRkLeaf* rk = nullptr;
  GemvSide side[2];                       // [0] 'N', [1] 'T' / 'C'
};

}  // namespace hmatb200
