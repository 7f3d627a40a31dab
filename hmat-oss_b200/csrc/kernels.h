// Host-side launch interface of the B200 engine's device phases.  Plain types only; the
// engine (engine.cu) owns the device buffers and calls these launchers on its stream.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace hmatb200 {

// One admissible leaf as the ACA and truncation phases see it.
struct RkLeafDesc {
  int row_off, m;     // rows [row_off, row_off + m) in cluster order
  int col_off, n;     // cols [col_off, col_off + n)
  long long ws_off;   // element offset of the leaf's slot in the ACA workspace
  long long fl_off;   // byte offset of the leaf's pivot flags (m + n bytes)
  int kcap;           // rank capacity of the slot
  int pad;
};
// Workspace slot layout (elements of T, from ws_off): A (m x kcap), B (n x kcap),
// aRef (m), bRef (n).
inline long long rk_slot_elems(int m, int n, int kcap) { return (long long)(m + n) * (kcap + 1); }

// A row panel of a leaf in the arena: rows [rs, rs + len) of the leaf (relative), stored
// column-major at `off` (len x n for full leaves, len x k for the A factor of Rk leaves).
struct PanelDesc {
  int rs, len;
  long long off;
};

// One dense (non-admissible) leaf and its row panels.
struct FullLeafDesc {
  int row_off, m, col_off, n;
  int panel_first, npanel;
};

// One piece of a segmented relayout (elements): a rows x cols column-major block, leading
// dimensions src_ld and dst_ld (a contiguous run is cols = 1).
struct CopySeg {
  long long src, dst;
  int rows, cols;
  int src_ld, dst_ld;
};
template <typename T>
void launch_copy_segments(const CopySeg* segs, int nseg, const T* src, T* dst, cudaStream_t s);

// Where the truncated factors of an Rk leaf go: A as row panels, B transposed (k x n).
struct RkStoreDesc {
  int panel_first, npanel;
  long long bt_off;
  int bt_ld;  // leading dimension of B^T (0: k, the leaf's own k x n block)
  int pad;
};

// ---- assembly ----
template <typename T>
void launch_assemble_full(const FullLeafDesc* d_leaves, int nleaves, const PanelDesc* panels, const KernelParams& kp,
                          Points pts, T* arena, cudaStream_t s);
// Full leaves from canonical payloads (m x n column-major at goff[leaf]) into arena panels.
template <typename T>
void launch_full_from_canonical(const FullLeafDesc* d_leaves, const long long* goff, int nleaves,
                                const PanelDesc* panels, const T* src, T* arena, cudaStream_t s);

// ACA+ (compression.cpp:553-724), delegating to partial ACA when n * 100 < m.  Leaves are
// taken in `order` from a device work counter that must be zero at launch.  `threads` is the
// CTA size: 64, 128, 256 or 512.  Every size builds the same factors (the Gram terms are summed a
// warp per term, pivot searches break ties by first index), so the size is a pure speed
// choice, made per leaf-size bucket by the engine's autotuner.
constexpr int kAcaBigRows = 2048;
template <typename T>
void launch_aca(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp, Points pts,
                double epsilon, T* ws, unsigned char* flags, int* ranks, int* status, int* counter, int kcap_max,
                int grid, cudaStream_t s, int threads = 128);
// Leaves in flight at once on the whole GPU: resident CTAs of `threads` (64 ... 512), or
// resident warps of the warp-per-leaf kernel for threads == 0, at rank capacity kcap_max.
template <typename T>
int aca_concurrency(int threads, int kcap_max);

// Warp-per-leaf ACA+ of the small leaves (m, n <= 64, not the partial-ACA delegate): same
// pivots and factors as launch_aca, the factors growing in shared memory.  Its rank
// capacity is min(slot capacity, 32 / 24 / 16 by scalar size); a leaf that needs more is
// reported as out of capacity.  Separate work counter.
bool aca_warp_eligible(int m, int n);
template <typename T>
void launch_aca_warp(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp,
                     Points pts, double epsilon, T* ws, int* ranks, int* status, int* counter, int kcap_max,
                     cudaStream_t s);

// Dense block written as an exact rank-min(m, n) factorisation, for the SVD compression
// of small blocks (the truncation phase then performs the SVD).
template <typename T>
void launch_dense_to_rk(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp,
                        Points pts, T* ws, int* ranks, int* status, cudaStream_t s);

// Multi-strata assembly (strata.cu): A[:, 0 .. rank) *= w in the slots of the leaves in order;
// the ks[b] columns of a stratum's factors (slot b of src, A scaled by w) appended after the
// kcur[b] columns of slot b of dst; the full block A B^T of the kcat[b] columns of the leaves in
// order (kcur[b] and the rest summed separately) written back as its exact rank-min(m, n)
// factorisation, through scratch (m x n at dof[item]).
template <typename T>
void launch_scale_a(const RkLeafDesc* d_leaves, const int* d_order, int count, const int* ranks, double w, T* ws,
                    cudaStream_t s);
template <typename T>
void launch_append_factors(const RkLeafDesc* src_desc, const RkLeafDesc* dst_desc, int nb, const int* kcur,
                           const int* ks, double w, const T* src, T* dst, cudaStream_t s);
template <typename T>
void launch_exact_factors(const RkLeafDesc* d_leaves, const int* d_order, int count, const int* kcur,
                          const int* kcat, const long long* dof, T* ws, T* scratch, cudaStream_t s);

// Truncation (rk_matrix.cpp:490-585): replaces A, B in each slot by the recompressed
// factors (first new-rank columns, same slot) and rewrites ranks.  `scratch` holds
// `grid` per-CTA FP64 slabs of `slab_elems` wide elements each.
template <typename T>
void launch_truncate(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, double epsilon, T* ws,
                     int* ranks, int* status, int* counter, typename Traits<T>::wide* scratch,
                     long long slab_elems, int grid, cudaStream_t s);
template <typename T>
long long truncate_slab_elems(int max_m, int max_n, int max_k);

// Arena panels of assembled Rk leaves back into workspace slots (inverse of launch_compact).
template <typename T>
void launch_unpack(const RkLeafDesc* d_leaves, int nleaves, const int* ranks, const RkStoreDesc* store,
                   const PanelDesc* panels, const T* arena, T* ws, cudaStream_t s);

// Copies the truncated factors of each leaf from its workspace slot into the arena:
// A as row panels, B transposed.
template <typename T>
void launch_compact(const RkLeafDesc* d_leaves, int nleaves, const T* ws, const int* ranks,
                    const RkStoreDesc* store, const PanelDesc* panels, T* arena, cudaStream_t s);

// Tall-skinny truncation (see truncate.cu): the triangular factors of A and B from row
// segments, the core SVD, and the new factors as A and B times small maps.
//
// One row segment of a factor (or one stack of segment triangles), reduced to a K x K
// triangle by the tsqr phase; the same list drives the apply phase.
struct TsItem {
  long long src;    // element offset of the segment's row 0, column 0 (ws, or the triangle buffer)
  long long r_out;  // element offset (wide) of the output triangle in the triangle buffer
  long long map;    // element offset (wide) of the factor's K x K map (apply phase)
  int rows, ld;     // rows of the segment; leading dimension of the source
  int ld_r;         // leading dimension of the output triangle
  int leaf, k;      // leaf (rank written by the core phase) and its rank before truncation
  int pad;
};
// One leaf of the core phase: its two K x K triangles and two K x K maps (ld K).
struct TsCore {
  long long ra, rb, ma, mb;
  int leaf, k;
};
// Largest rank the tall-skinny path takes (32 real, 16 complex), and the rank bucket
// (8, 16, 24 or 32) of rank k (0 when above the largest).
template <typename T>
int ts_kmax();
int ts_bucket(int k, int kmax);
constexpr int kTsSegRows = 512;  // rows per segment
template <typename T>
void launch_tsqr(int K, const TsItem* items, int nitems, const T* ws, typename Traits<T>::wide* tri,
                 bool from_tri, cudaStream_t s);
template <typename T>
void launch_tscore(int K, const TsCore* items, int nitems, const typename Traits<T>::wide* tri,
                   typename Traits<T>::wide* maps, int* ranks, int* status, double eps, cudaStream_t s);
template <typename T>
void launch_tsapply(int K, const TsItem* items, int nitems, T* ws, const typename Traits<T>::wide* maps,
                    const int* ranks, cudaStream_t s);
// The same phases for ranks above the register buckets: a CTA per item with an FP64 slab of
// `slab` wide elements per CTA (tsqr: rows x k + k + k^2; core: 2 k^2 + 2 k; apply: rows x k'
// scalars), `grid` CTAs, one work counter.
template <typename T>
void launch_tsqr_cta(const TsItem* items, int nitems, const T* ws, typename Traits<T>::wide* tri, bool from_tri,
                     typename Traits<T>::wide* scratch, long long slab, int grid, int* counter, cudaStream_t s);
template <typename T>
void launch_tscore_cta(const TsCore* items, int nitems, const typename Traits<T>::wide* tri,
                       typename Traits<T>::wide* maps, int* ranks, int* status, double eps,
                       typename Traits<T>::wide* scratch, long long slab, int grid, int* counter, cudaStream_t s);
template <typename T>
void launch_tsapply_cta(const TsItem* items, int nitems, T* ws, const typename Traits<T>::wide* maps,
                        const int* ranks, typename Traits<T>::wide* scratch, long long slab, int grid, int* counter,
                        cudaStream_t s);

// ---- gemv ----
}  // namespace hmatb200
#include "gemv_plan.h"
namespace hmatb200 {
// y = alpha op(H) x + beta y on device buffers (client numbering); `xz` is the scratch
// buffer of plan.xz_rows rows of gemv_rhs_stride(sizeof(T), 16) scalars; `err` is set when
// a pipeline wait gives up.
template <typename T>
void launch_gemv(const GemvPlan& p, char trans, int nrhs, T alpha, T beta, const T* x_client, T* y_client, T* xz,
                 GemvStatus* err, cudaStream_t s, const GemvTiming* timing = nullptr);
// Row stride (scalars) of the xz buffer for R right-hand sides.
int gemv_rhs_stride(int elem_bytes, int R);
// Kernel launches of one product with nrhs right-hand sides.
int gemv_launch_count(const GemvPlan& p, char trans, int nrhs, int elem_bytes);
// Dynamic shared memory of one streamed-task CTA, and of one warp-level CTA (and its warps).
size_t stream_smem_bytes(int elem_bytes, int R, int RS, int omax, bool transposed);
size_t warp_stream_smem_bytes(int elem_bytes);
size_t umma_smem_bytes();
int warp_stream_warps_per_cta();
// Resident CTAs an SM of the tensor-core gemv kernel (FP32 or FP64) with `ntile` 8-row tiles
// (its register budget).
int mma_stream_blocks_per_sm(int ntile, int elem_bytes);

// Leaf-factor gradients of y = H x for the output gradient r (real types; x, r device,
// client numbering, nrhs <= 16): dF = r_I x_J^T, dA = r_I (B^T x_J)^T, dB = x_J (A^T r_I)^T,
// written (or added) into gradient arenas laid out like the leaf arenas.
template <typename T>
void launch_leaf_gradients(const GemvPlan& p, int nrhs, const T* x, const T* r, T* xz, T* rz, T* gfull, T* grk,
                           bool accumulate, GemvStatus* err, cudaStream_t s);
// dx = H^T r and the leaf gradients of y = H x at the output gradient r, in one pass (the
// transposed product's z' = A^T r serves both); nrhs <= 16.
template <typename T>
void launch_gemv_adjoint(const GemvPlan& p, int nrhs, const T* x, const T* r, T* dx, T* xz, T* rz, T* gfull, T* grk,
                         bool accumulate, GemvStatus* err, cudaStream_t s);

// Load the assembly kernels of the storage type T ahead of the first assembly.
template <typename T>
void preload_aca_kernels();
template <typename T>
void preload_full_kernels();
template <typename T>
void preload_truncate_kernels();
// Cap on the one-sided Jacobi sweeps of the truncation's core SVDs, for the device that is
// current (default kJacobiDefaultSweeps).
constexpr int kJacobiDefaultSweeps = 60;
cudaError_t set_jacobi_max_sweeps(int sweeps);

// Grid size of a persistent launch: a multiple of the SM count.
int persistent_grid(int blocks_per_sm);

}  // namespace hmatb200
