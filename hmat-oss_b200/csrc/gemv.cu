// Batched H-matrix-vector product over all leaves (sm_100a).
//
// Restates HMatrix<T>::gemv (h_matrix.cpp:792-857) with its leaf products
// (ScalarArray::gemm, scalar_array.cpp:413-443; RkMatrix::gemv, rk_matrix.cpp:156-206) and the
// reorderVector / restoreVectorOrder permutations of the C wrapper (h_matrix.cpp:75-141,
// c_wrapping.hpp:233-252), as a few launches over device-resident schedules (gemv_plan.h):
//
//   gather   xz[i][q] = x[perm[i] + q ld]           client -> cluster order, row-major
//   z-phase  z_L = B_L^T x_J ('N') / A_L^T x_I ('T')  one task per Rk leaf (chunks for long ones)
//   z-reduce sums the chunk partials of long leaves
//   y-phase  y_I = beta y_I + alpha sum (F x | A z)   one task per output block; the result is
//                                                     scattered straight to client order
//
// Every task streams its units (contiguous pieces of the leaf arena and of the xz buffer)
// through a shared-memory pipeline filled by TMA bulk copies (cp.async.bulk, completion on
// an mbarrier), on a persistent grid where each CTA owns a contiguous range of tasks of
// about equal bytes.  Each thread accumulates up to 4 output rows x R right-hand sides in
// registers; inner-dimension slices (warps, and lanes when the output is narrow) are summed
// at the end of each task in a fixed order, so repeated products are bitwise identical.
#include <type_traits>

#include "gemv_plan.h"
#include "kernels.h"

namespace hmatb200 {
size_t warp_stream_smem_bytes(int elem_bytes);
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kPieceCols = 32;         // inner extent of a non-transposed unit
constexpr int kPieceElems = 128 * 32;  // P capacity of a stage (elements)
constexpr int kMaxInner = 128;         // inner extent of a transposed unit

// ---------------------------------------------------------------------------------
// TMA bulk copy + mbarrier helpers
__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Programmatic dependent launch.  The kernels after the gather in a product are launched with
// programmatic stream serialization (launch_pdl) and start with pdl_wait(), which returns once
// the kernel before them on the stream has completed and its writes are visible (for a kernel
// launched normally it returns at once).  No kernel triggers its dependents early: their launch
// then overlaps only the end of the kernel before them (100,000-point cylinder, FP32, graph
// replay: 0.250 -> 0.247 ms).  Triggering at the start of every kernel let the next grid be
// scheduled beside the persistent kernels and took the product to 0.285 ms.
__device__ inline void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ inline void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ inline void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ inline void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// L2 policies of the streamed copies: a leaf piece is read once per product (evict first), the
// x / z rows by every unit over their columns (evict last), so that the stream of pieces does
// not push the vector rows out of L2 and the units read them from DRAM again (100,000-point
// cylinder, 16 right-hand sides: FP32 product 0.248 -> 0.2435 ms, FP64 0.750 -> 0.743 ms).
__device__ inline uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ inline uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ inline void bulk_g2s_hint(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}
// A leaf piece, and the X rows of a unit.
__device__ inline void bulk_piece(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  bulk_g2s_hint(dst, src, bytes, bar, policy_evict_first());
}
__device__ inline void bulk_xrows(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  bulk_g2s_hint(dst, src, bytes, bar, policy_evict_last());
}
__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for a barrier phase: false once `limit` polls went by without it completing.
// A negative limit gives up at once (a test mode of the status path: the caller still drains
// its copies with a positive limit before it stops).
__device__ inline bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit) {
  if (limit < 0) return false;
  long long spins = 0;
  while (!mbar_try_wait(bar, parity))
    if (++spins > limit) return false;
  return true;
}

// A warp whose wait gave up: sets the status flag, then waits (bounded) for the copies of
// the units it has issued and not consumed (u .. last_issued, one stage each) to land, so
// that no bulk copy is still writing its shared memory when it exits.
__device__ inline long long drain_limit(const GemvStatus* st) {
  return st->wait_limit > 0 && st->wait_limit < kGemvDrainLimit ? st->wait_limit : kGemvDrainLimit;
}
__device__ inline void warp_give_up(GemvStatus* st, uint64_t* bars, int nstages, int u_begin, int u, int last_issued) {
  atomicCAS(&st->failed, 0, 1);
  const long long lim = drain_limit(st);
  for (int v = u; v <= last_issued; ++v)
    mbar_wait_bounded(&bars[(v - u_begin) % nstages], (uint32_t)(((v - u_begin) / nstages) & 1), lim);
}

__device__ inline uint32_t round16(uint64_t b) { return (uint32_t)((b + 15) & ~15ull); }

__device__ inline float shfl_xor(float v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ inline double shfl_xor(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ inline cfloat shfl_xor(cfloat v, int m) {
  return cfloat{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}
__device__ inline cdouble shfl_xor(cdouble v, int m) {
  return cdouble{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}

// Loads Q consecutive elements from shared memory (vectorised when aligned).
template <typename T, int Q>
__device__ inline void lds_vec(const T* p, T (&out)[Q]) {
  constexpr int bytes = Q * (int)sizeof(T);
  if constexpr (bytes % 16 == 0) {
    const uint4* s = reinterpret_cast<const uint4*>(p);
    uint4* d = reinterpret_cast<uint4*>(out);
#pragma unroll
    for (int c = 0; c < bytes / 16; ++c) d[c] = s[c];
  } else if constexpr (bytes % 8 == 0) {
    const uint2* s = reinterpret_cast<const uint2*>(p);
    uint2* d = reinterpret_cast<uint2*>(out);
#pragma unroll
    for (int c = 0; c < bytes / 8; ++c) d[c] = s[c];
  } else {
#pragma unroll
    for (int c = 0; c < Q; ++c) out[c] = p[c];
  }
}

template <typename T>
constexpr int rs_of(int R) {
  return R * (int)sizeof(T) >= 16 ? R : (16 / (int)sizeof(T));
}
template <typename T>
constexpr int nstage_of() {
  return sizeof(T) >= 16 ? 2 : 3;
}

// ---------------------------------------------------------------------------------
// x (client order, column-major with leading dimension ldx; right-hand sides q0 .. q0 + R - 1
// of r) into xz in cluster order (row-major, RS columns, zeros past R).  A CTA takes
// kGatherRows client rows: it reads each column of x along the rows (coalesced), transposes
// through shared memory, and writes each client row's RS values as one contiguous xz row at
// its cluster position iperm[j].  One more CTA clears the kZeroRows zero rows from row `zrow0`
// (the X rows of the y matrices' padding columns) and the ncnt chunk counters of the fused z
// sums, so that every product starts from zero (also after one that stopped early).
constexpr int kGatherRows = 64;
template <typename T, int R, int RS>
__global__ void __launch_bounds__(256) gather_kernel(const T* __restrict__ x, int N, int ldx, int q0, int r,
                                                     const int* __restrict__ iperm, T* __restrict__ xz, int zrow0,
                                                     int* zcnt, int ncnt) {
  __shared__ T tile[RS][kGatherRows + 1];
  const int nblk = (N + kGatherRows - 1) / kGatherRows;
  if ((int)blockIdx.x >= nblk) {
    for (int e = threadIdx.x; e < kZeroRows * RS; e += blockDim.x) xz[(size_t)zrow0 * RS + e] = zero<T>();
    for (int e = threadIdx.x; e < ncnt; e += blockDim.x) zcnt[e] = 0;  // the z sums' chunk counters
    return;
  }
  const int j0 = blockIdx.x * kGatherRows;
  for (int e = threadIdx.x; e < RS * kGatherRows; e += blockDim.x) {
    const int q = e / kGatherRows, jl = e % kGatherRows, j = j0 + jl;
    T v = zero<T>();
    if (j < N && q < R && q0 + q < r) v = x[(size_t)j + (size_t)(q0 + q) * ldx];
    tile[q][jl] = v;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < RS * kGatherRows; e += blockDim.x) {
    const int jl = e / RS, q = e % RS, j = j0 + jl;
    if (j < N) xz[(size_t)iperm[j] * RS + q] = tile[q][jl];
  }
}
inline unsigned gather_grid(int N) { return (unsigned)((N + kGatherRows - 1) / kGatherRows + 1); }

// Loads through L2 only (another SM's writes, made visible by its fence, are not in this
// SM's L1).
__device__ inline float ld_l2(const float* p) { return __ldcg(p); }
__device__ inline double ld_l2(const double* p) { return __ldcg(p); }
__device__ inline cfloat ld_l2(const cfloat* p) {
  const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
  return cfloat{v.x, v.y};
}
__device__ inline cdouble ld_l2(const cdouble* p) {
  const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
  return cdouble{v.x, v.y};
}

// End of a z task that is a chunk of a long group (task.red >= 0), after its partial slot is
// written: the warp's writes are fenced, the sum's counter taken, and the warp that finishes
// the sum's last chunk adds the partial slots in part order into the final slot (the order of
// zred_kernel, so the result does not depend on which chunk finishes last).  No warp waits.
template <typename T, int RS>
__device__ inline void z_chunk_done(const GemvTask& task, const GemvZred* __restrict__ zred, int* zcnt, T* xz,
                                    int lane) {
  if (task.red < 0 || !zcnt) return;
  __threadfence();
  __syncwarp();
  int last = 0;
  if (lane == 0) last = atomicAdd(&zcnt[task.red], 1) == zred[task.red].nparts - 1;
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __threadfence();
  const GemvZred d = zred[task.red];
  for (int e = lane; e < d.k * RS; e += 32) {
    T v = zero<T>();
    for (int p = 0; p < d.nparts; ++p) v = v + ld_l2(xz + ((size_t)d.part_row + (size_t)p * d.k) * RS + e);
    xz[(size_t)d.final_row * RS + e] = v;
  }
}

// Checks a unit's copies into a warp-level stage before they are issued: 16-byte sizes and
// addresses (the bulk-copy rule), the piece below the X rows, the X rows inside the stage, and
// runs that cover exactly its columns.  A unit that fails is not copied: the stage's barrier
// gets a plain arrival (so nothing waits for it), and the status block records code 2 and the
// unit's index.
template <typename T, int RS>
__device__ inline bool unit_copies_ok(const GemvUnit& U, const T* arena, const T* xz, int stage_bytes, int xoff) {
  const uint64_t pbytes = round16((uint64_t)U.pel * sizeof(T));
  const uint64_t xbytes = (uint64_t)U.c * RS * sizeof(T);
  if (U.c <= 0 || U.pel <= 0 || (reinterpret_cast<uintptr_t>(arena + U.poff) & 15) != 0) return false;
  if (xoff < (int)pbytes || xoff % 16 != 0 || (uint64_t)xoff + xbytes > (uint64_t)stage_bytes) return false;
  if (((size_t)RS * sizeof(T)) % 16 != 0) return false;
  if (U.nruns < 0 || U.nruns > kUnitRuns) return false;
  if (U.nruns > 0) {
    int rows = 0;
    for (int r = 0; r < kUnitRuns; ++r)
      if (r < U.nruns) rows += U.run_len[r];
    if (rows != U.c) return false;
  }
  return true;
}
__device__ inline void record_bad_unit(GemvStatus* st, int u) {
  atomicExch(&st->failed, 2);
  atomicExch(&st->pad, u);
}

// The X rows of a unit into a pipeline stage: one bulk copy, or one per run.
template <typename T, int RS>
__device__ inline void issue_x(unsigned char* dst, const T* xz, const GemvUnit& U, uint64_t* bar) {
  if (U.nruns == 0) {
    bulk_xrows(dst, xz + (size_t)U.xrow * RS, (uint32_t)U.c * RS * (uint32_t)sizeof(T), bar);
    return;
  }
  uint32_t off = 0;
#pragma unroll
  for (int r = 0; r < kUnitRuns; ++r) {  // constant indices: the descriptor stays in registers
    if (r < U.nruns) {
      const uint32_t b = (uint32_t)U.run_len[r] * RS * (uint32_t)sizeof(T);
      bulk_xrows(dst + off, xz + (size_t)U.run_row[r] * RS, b, bar);
      off += b;
    }
  }
}

// ---------------------------------------------------------------------------------
// The streamed task kernel.  OL output lanes x (32 / OL) inner slices per warp, RPT rows per
// lane (output rows <= OL * RPT), R right-hand sides (xz row stride RS).
template <typename T, int R, int RS, int OL, int RPT, bool TRANSP, int NSTAGE>
__global__ void __launch_bounds__(kThreads) stream_kernel(const GemvTask* __restrict__ tasks,
                                                          const int* __restrict__ cta_begin,
                                                          const GemvUnit* __restrict__ units,
                                                          const T* __restrict__ arena, T* xz, int conj,
                                                          int out_is_y, const int* __restrict__ perm_out,
                                                          T* __restrict__ y, int ldy, int q0, int r, T alpha,
                                                          T beta, GemvStatus* err) {
  constexpr int LS = 32 / OL;
  constexpr int OMAX = OL * RPT;
  constexpr int XCAP = (TRANSP ? kMaxInner : kPieceCols) * RS;
  constexpr int PCAP = kPieceElems + 2 * OMAX + 16;  // slack: alignment shift, masked lanes reading past a piece
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* Ps = reinterpret_cast<T*>(smem_raw);
  T* Xs = Ps + (size_t)NSTAGE * PCAP;
  T* red = Xs + (size_t)NSTAGE * XCAP;
  uint64_t* bars = reinterpret_cast<uint64_t*>(red + (size_t)kWarps * OMAX * R);

  const int t0 = cta_begin[blockIdx.x], t1 = cta_begin[blockIdx.x + 1];
  if (t0 >= t1) return;
  const int u_begin = tasks[t0].first_unit;
  const int u_end = tasks[t1 - 1].first_unit + tasks[t1 - 1].nunits;
  const long long wlim = err->wait_limit;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ol = lane % OL, ls = lane / OL;

  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // producer: thread 0 arms a stage's barrier and issues the unit's two bulk copies
  auto issue = [&](int u) {
    const int s = (u - u_begin) % NSTAGE;
    const GemvUnit U = units[u];
    // the copy starts at the 16-byte boundary at or below the piece (TMA alignment rule)
    const uint32_t pbytes = round16((uint64_t)(U.pel + U.shift) * sizeof(T));
    const uint32_t xbytes = (uint32_t)U.c * RS * (uint32_t)sizeof(T);
    mbar_expect_tx(&bars[s], pbytes + xbytes);
    bulk_piece(Ps + (size_t)s * PCAP, arena + (U.poff - U.shift), pbytes, &bars[s]);
    bulk_xrows(Xs + (size_t)s * XCAP, xz + (size_t)U.xrow * RS, xbytes, &bars[s]);
  };
  if (tid == 0)
    for (int u = u_begin; u < u_end && u < u_begin + NSTAGE; ++u) issue(u);

  int u = u_begin;
  for (int t = t0; t < t1; ++t) {
    const GemvTask task = tasks[t];
    T acc[RPT][R];
#pragma unroll
    for (int a = 0; a < RPT; ++a)
#pragma unroll
      for (int q = 0; q < R; ++q) acc[a][q] = zero<T>();

    for (int k = 0; k < task.nunits; ++k, ++u) {
      const int s = (u - u_begin) % NSTAGE;
      const uint32_t parity = (uint32_t)(((u - u_begin) / NSTAGE) & 1);
      const bool ok = mbar_wait_bounded(&bars[s], parity, wlim);
      const GemvUnit U = units[u];
      const T* P = Ps + (size_t)s * PCAP + U.shift;
      const T* X = Xs + (size_t)s * XCAP;
      const int c = U.c;
      if constexpr (!TRANSP) {
        // P is O x c column-major: out[o] += sum_j P[o, j] X[j]
        const int O = task.O;
#pragma unroll 2
        for (int j = warp * LS + ls; j < c; j += kWarps * LS) {
          T xv[R];
          lds_vec<T, R>(X + (size_t)j * RS, xv);
#pragma unroll
          for (int a = 0; a < RPT; ++a) {
            const T p = P[ol + a * OL + (size_t)j * O];
#pragma unroll
            for (int q = 0; q < R; ++q) acc[a][q] = fmadd(p, xv[q], acc[a][q]);
          }
        }
      } else {
        // P is c x ow column-major, covering outputs [o0, o0 + ow):
        // out[o] += sum_j op(P[j, o - o0]) X[j]
        const int o0 = U.o0, ow = U.ow;
        for (int j = warp * LS + ls; j < c; j += kWarps * LS) {
          T xv[R];
          lds_vec<T, R>(X + (size_t)j * RS, xv);
#pragma unroll
          for (int a = 0; a < RPT; ++a) {
            const int oo = ol + a * OL - o0;
            if (oo >= 0 && oo < ow) {
              T p = P[j + (size_t)oo * c];
              if (conj) p = conjg(p);
#pragma unroll
              for (int q = 0; q < R; ++q) acc[a][q] = fmadd(p, xv[q], acc[a][q]);
            }
          }
        }
      }
      // stage s is free again; a copy that did not land in time stops the whole CTA, after
      // the copies it has in flight (units u .. u + NSTAGE - 1) have landed
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicCAS(&err->failed, 0, 1);
          for (int v = u; v < u_end && v < u + NSTAGE; ++v)
            mbar_wait_bounded(&bars[(v - u_begin) % NSTAGE], (uint32_t)(((v - u_begin) / NSTAGE) & 1),
                              drain_limit(err));
        }
        return;
      }
      if (tid == 0 && u + NSTAGE < u_end) issue(u + NSTAGE);
    }

    // ---- epilogue: lane slices, then warps, in a fixed order ----
#pragma unroll
    for (int m = OL; m < 32; m <<= 1)
#pragma unroll
      for (int a = 0; a < RPT; ++a)
#pragma unroll
        for (int q = 0; q < R; ++q) acc[a][q] = acc[a][q] + shfl_xor(acc[a][q], m);
    if (ls == 0) {
#pragma unroll
      for (int a = 0; a < RPT; ++a)
#pragma unroll
        for (int q = 0; q < R; ++q) red[((size_t)warp * OMAX + ol + a * OL) * R + q] = acc[a][q];
    }
    __syncthreads();
    for (int e = tid; e < task.O * R; e += kThreads) {
      const int o = e / R, q = e % R;
      T v = red[(size_t)o * R + q];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) v = v + red[((size_t)w * OMAX + o) * R + q];
      if (out_is_y) {
        if (q0 + q < r) {
          T* yp = y + (size_t)perm_out[task.out_row + o] + (size_t)(q0 + q) * ldy;
          T outv = alpha * v;
          if (!is_zero_val(beta)) outv = fmadd(beta, *yp, outv);
          *yp = outv;
        }
      } else {
        xz[(size_t)(task.out_row + o) * RS + q] = v;
      }
    }
    if constexpr (RS > R) {
      if (!out_is_y)
        for (int e = tid; e < task.O * (RS - R); e += kThreads)
          xz[(size_t)(task.out_row + e / (RS - R)) * RS + R + e % (RS - R)] = zero<T>();
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------
// The descriptors of the next unit and the next task a warp-level kernel issues, prefetched one
// issue ahead.  LANES = true spreads each over the warp's lanes, one 32-bit word a lane, and
// gathers it with shuffles when it is used (every lane calls get()), instead of holding it whole
// in every lane's registers through the unit's sums.  The FP64 y-phase kernel then keeps its
// accumulators without spilling (100,000-point cylinder, 16 right-hand sides: y-phase 0.393 ->
// 0.340 ms) and the FP32 one with up to 8 tiles schedules better (0.128 -> 0.1245 ms); the
// column-slice z kernels keep the whole copy (the FP64 one is slower with the shuffles, 0.349 ->
// 0.362 ms), and so does the 16-tile FP32 kernel (it spills more with them).
constexpr int kUnitWords = (int)(sizeof(GemvUnit) / 4);
constexpr int kTaskWords = (int)(sizeof(GemvTask) / 4);
static_assert(sizeof(GemvUnit) % 4 == 0 && kUnitWords <= 32, "unit descriptor words");
static_assert(sizeof(GemvTask) % 4 == 0 && kTaskWords <= 32, "task descriptor words");
template <typename D, int W>
__device__ __forceinline__ D from_lanes(uint32_t w) {
  D d;
  uint32_t* p = reinterpret_cast<uint32_t*>(&d);
#pragma unroll
  for (int i = 0; i < W; ++i) p[i] = __shfl_sync(0xffffffffu, w, i);
  return d;
}
template <bool LANES>
struct NextUnit {  // lane 0 holds the descriptor
  GemvUnit d;
  __device__ void load(const GemvUnit* units, int v, int lane) {
    if (lane == 0) d = units[v];
  }
  __device__ GemvUnit get() const { return d; }
};
template <>
struct NextUnit<true> {  // lane l < kUnitWords holds word l
  uint32_t w = 0;
  __device__ void load(const GemvUnit* units, int v, int lane) {
    w = lane < kUnitWords ? __ldg(reinterpret_cast<const uint32_t*>(units + v) + lane) : 0u;
  }
  __device__ GemvUnit get() const { return from_lanes<GemvUnit, kUnitWords>(w); }
};
template <bool LANES>
struct NextTask {  // every lane holds the descriptor
  GemvTask d;
  __device__ void load(const GemvTask* tasks, int t, int /*lane*/) { d = tasks[t]; }
  __device__ GemvTask get() const { return d; }
};
template <>
struct NextTask<true> {  // lane l < kTaskWords holds word l
  uint32_t w = 0;
  __device__ void load(const GemvTask* tasks, int t, int lane) {
    w = lane < kTaskWords ? __ldg(reinterpret_cast<const uint32_t*>(tasks + t) + lane) : 0u;
  }
  __device__ GemvTask get() const { return from_lanes<GemvTask, kTaskWords>(w); }
};

// ---------------------------------------------------------------------------------
// Warp-level streamed tasks (the 'N' products).  Every warp owns a contiguous range of whole
// tasks and runs its own two-stage TMA pipeline: lane 0 copies the unit descriptor into the
// stage and issues the unit's bulk copies (P piece; X rows at the unit's byte offset o0 in the
// stage, right after the piece), completion on the stage's
// mbarrier, so warps never wait for one another.  Lane maps (output rows O of the task):
//   MODE 2 (O <= 32): the warp is a window of floor(32 / O) column slices x O rows, lane =
//          slice * O + row; P is read as one contiguous run per step (no bank conflicts);
//          the slices are summed through shared memory at the end of the task.
//   MODE 1 (O <= 16 * A2): two column slices (half-warps) x 16 rows, A2 rows per lane
//          (row, row + 16, ...); slices summed with one shuffle.
//   MODE 0 (O <= 32 * A2): lanes over rows, A2 rows per lane, one slice.
// Row groups above O are skipped warp-uniformly.  Every lane keeps all R right-hand sides
// of its rows; float sums use the paired FMA (fma.rn.f32x2: two IEEE fmaf per
// instruction).  Summation orders are fixed, so repeated products are bitwise identical.
constexpr int kWarpCTA = 4;
constexpr int kWarpStages = 2;
__host__ __device__ constexpr int warp_stage_bytes(int elem_bytes) { return warp_piece_bytes(elem_bytes) + kWarpXBytes; }

// R accumulators of one output row, and one X row as the FMAs consume it.
template <typename T, int R, bool PAIR = std::is_same<T, float>::value && (R % 2 == 0)>
struct RowOps {
  using XV = T[R];
  using AV = T[R];
  __device__ static void load(const T* p, XV& x) { lds_vec<T, R>(p, x); }
  __device__ static void zero_(AV& a) {
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = zero<T>();
  }
  __device__ static void fma(T p, const XV& x, AV& a) {
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = fmadd(p, x[q], a[q]);
  }
  __device__ static T get(const AV& a, int q) { return a[q]; }
};
template <int R>
struct RowOps<float, R, true> {
  static constexpr int N = R / 2;
  using XV = unsigned long long[N];
  using AV = unsigned long long[N];
  __device__ static void load(const float* p, XV& x) {
    if constexpr (R % 4 == 0) {
      const ulonglong2* s = reinterpret_cast<const ulonglong2*>(p);
#pragma unroll
      for (int c = 0; c < R / 4; ++c) {
        const ulonglong2 v = s[c];
        x[2 * c] = v.x;
        x[2 * c + 1] = v.y;
      }
    } else {
      const unsigned long long* s = reinterpret_cast<const unsigned long long*>(p);
#pragma unroll
      for (int c = 0; c < N; ++c) x[c] = s[c];
    }
  }
  __device__ static void zero_(AV& a) {
#pragma unroll
    for (int i = 0; i < N; ++i) a[i] = 0ull;  // the bits of (+0.0f, +0.0f)
  }
  __device__ static void fma(float p, const XV& x, AV& a) {
    unsigned long long pp;
    asm("mov.b64 %0, {%1, %1};" : "=l"(pp) : "f"(p));
#pragma unroll
    for (int i = 0; i < N; ++i) asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(a[i]) : "l"(pp), "l"(x[i]));
  }
  __device__ static float get(const AV& a, int q) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a[q / 2]));
    return (q & 1) ? hi : lo;
  }
};

// One unit of a warp task: lane's rows row0 + a * stride (a < NA) of the columns
// j = js, js + SL, ... < c, all R right-hand sides.
// O is the column stride of the piece.  With `active` >= 0 only the first `active` row
// groups are computed (a guarded loop).
// UNROLL: columns a loop iteration takes (4 for the lanes-over-rows maps, 1 for the
// column-slice windows: FP64 y-phase 0.345 -> 0.331 ms, z-phase 0.334 -> 0.333 ms against 2 for
// both on the 100,000-point cylinder, 16 right-hand sides).
template <typename T, int R, int RS, int NA, int A2, int UNROLL>
__device__ __forceinline__ void rows_loop(const T* P, const T* X, int c, int js, int SL, int O, int row0, int stride,
                                          typename RowOps<T, R>::AV (&acc)[A2], int active = -1) {
  using Ops = RowOps<T, R>;
#pragma unroll UNROLL
  for (int j = js; j < c; j += SL) {
    typename Ops::XV xv;
    Ops::load(X + (size_t)j * RS, xv);
    const T* pc = P + (size_t)j * O + row0;
#pragma unroll
    for (int a = 0; a < NA; ++a)
      if (active < 0 || a < active) Ops::fma(pc[a * stride], xv, acc[a]);
  }
}

// Blocks per SM the register budget allows: more accumulator bytes, fewer resident warps.
template <typename T, int R, int A2>
constexpr int warp_min_blocks() {
  return A2 * R * (int)sizeof(T) <= 256 ? 4 : 2;
}

template <typename T, int R, int RS, int MODE, int A2>
__global__ void __launch_bounds__(kWarpCTA * 32, (warp_min_blocks<T, R, A2>()))
    warp_stream_kernel(const GemvTask* __restrict__ tasks, const int* __restrict__ warp_begin,
                       const GemvUnit* __restrict__ units, const T* __restrict__ arena, T* xz, GemvStatus* err,
                       const GemvZred* __restrict__ zred, int* zcnt) {
  using Ops = RowOps<T, R>;
  constexpr int OL = MODE == 0 ? 32 : 16;
  // MODE 2: right-hand sides per round of the slice sums (a power of two)
  constexpr int QC0 = warp_piece_bytes((int)sizeof(T)) / (32 * A2 * (int)sizeof(T));
  constexpr int QC1 = QC0 >= 16 ? 16 : (QC0 >= 8 ? 8 : (QC0 >= 4 ? 4 : (QC0 >= 2 ? 2 : 1)));
  constexpr int QC = QC1 < R ? QC1 : R;
  static_assert(QC >= 1 && (R % QC) == 0, "reduction chunk");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  pdl_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* wbase = smem_raw + (size_t)warp * kWarpStages * warp_stage_bytes((int)sizeof(T));
  // per stage: the unit's column count and X offset (what the consumers read), then the barriers
  int2* uslot =
      reinterpret_cast<int2*>(smem_raw + (size_t)kWarpCTA * kWarpStages * warp_stage_bytes((int)sizeof(T))) + warp * kWarpStages;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kWarpCTA * kWarpStages *
                                                               (warp_stage_bytes((int)sizeof(T)) + sizeof(int2))) +
                   warp * kWarpStages;
  const int gw = blockIdx.x * kWarpCTA + warp;
  const int t0 = warp_begin[gw], t1 = warp_begin[gw + 1];
  if (t0 >= t1) return;
  const int u_begin = tasks[t0].first_unit;
  const int u_end = tasks[t1 - 1].first_unit + tasks[t1 - 1].nunits;
  const long long wlim = err->wait_limit;

  if (lane == 0) {
    for (int s = 0; s < kWarpStages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncwarp();
  // lane 0: descriptor into the stage, then the unit's two bulk copies.  The descriptor of
  // the next unit to issue is loaded one issue ahead, off the critical path.
  constexpr bool kLanes = MODE != 2;
  NextUnit<kLanes> nxt;
  int last_issued = u_begin - 1;  // lane 0: the last unit whose copies were issued
  auto issue = [&](int u, const GemvUnit& U) {
    const int s = (u - u_begin) % kWarpStages;
    last_issued = u;
    uslot[s] = make_int2(U.c, U.o0);
    const uint32_t pbytes = round16((uint64_t)U.pel * sizeof(T));
    const uint32_t xbytes = (uint32_t)U.c * RS * (uint32_t)sizeof(T);
    unsigned char* st = wbase + (size_t)s * warp_stage_bytes((int)sizeof(T));
    if (!unit_copies_ok<T, RS>(U, arena, xz, warp_stage_bytes((int)sizeof(T)), U.o0)) {
      record_bad_unit(err, u);
      mbar_arrive(&bars[s]);
      return;
    }
    mbar_expect_tx(&bars[s], pbytes + xbytes);
    bulk_piece(st, arena + U.poff, pbytes, &bars[s]);
    issue_x<T, RS>(st + U.o0, xz, U, &bars[s]);
  };
  auto issue_next = [&](int v) {  // nxt holds units[v]; kLanes: every lane calls it, else lane 0
    const GemvUnit U = nxt.get();
    if (lane == 0) issue(v, U);
    if (v + 1 < u_end) nxt.load(units, v + 1, lane);
  };
  if (lane == 0)
    for (int v = u_begin; v < u_end && v < u_begin + kWarpStages; ++v) issue(v, units[v]);
  if (u_begin + kWarpStages < u_end) nxt.load(units, u_begin + kWarpStages, lane);

  int u = u_begin;
  NextTask<kLanes> task_next;
  task_next.load(tasks, t0, lane);
  for (int t = t0; t < t1; ++t) {
    const GemvTask task = task_next.get();
    if (t + 1 < t1) task_next.load(tasks, t + 1, lane);
    const int O = task.O;
    int row0, js, SL, Og = O;
    float inv = 1.f;
    if constexpr (MODE == 2) {
      // window: Og = ceil(O / A2) lanes per column, SL = floor(32 / Og) columns per step;
      // exact for lane < 32 and Og <= 32 (the quotients are at least 1/64 from integers)
      Og = (O + A2 - 1) / A2;
      inv = __frcp_rn((float)Og);
      SL = (int)(32.5f * inv);
      js = (int)(((float)lane + 0.5f) * inv);
      row0 = lane - js * Og;
    } else if constexpr (MODE == 1) {
      SL = 2;
      row0 = lane & 15;
      js = lane >> 4;
    } else {
      SL = 1;
      row0 = lane;
      js = 0;
    }
    // row groups holding rows of this task (warp-uniform)
    const int na = MODE == 2 ? A2 : min(A2, (O + OL - 1) / OL);
    typename Ops::AV acc[A2];
#pragma unroll
    for (int a = 0; a < A2; ++a) Ops::zero_(acc[a]);

    int s = 0;
    for (int kk = 0; kk < task.nunits; ++kk, ++u) {
      s = (u - u_begin) % kWarpStages;
      const uint32_t parity = (uint32_t)(((u - u_begin) / kWarpStages) & 1);
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[s], parity, wlim))) {
        // a copy did not land in time: flag it, let the copies in flight land, stop the warp
        if (lane == 0) warp_give_up(err, bars, kWarpStages, u_begin, u, last_issued);
        return;
      }
      const int c = uslot[s].x;
      const T* P = reinterpret_cast<const T*>(wbase + (size_t)s * warp_stage_bytes((int)sizeof(T)));
      const T* X = reinterpret_cast<const T*>(wbase + (size_t)s * warp_stage_bytes((int)sizeof(T)) + uslot[s].y);
      // Rows of a lane past O read the next column (or, in the last column, the first
      // elements of the X rows of the same stage); they are never written.
      if constexpr (MODE == 2) {
        if (js < SL) rows_loop<T, R, RS, A2, A2, 1>(P, X, c, js, SL, O, row0, Og, acc);
      } else {
        rows_loop<T, R, RS, A2, A2, 4>(P, X, c, js, SL, O, row0, OL, acc, na);
      }
      __syncwarp();  // every lane is done with stage s
      // the last unit's stage stays free until the epilogue has used it as scratch
      if ((kLanes || lane == 0) && kk + 1 < task.nunits && u + kWarpStages < u_end) issue_next(u + kWarpStages);
    }

    // ---- epilogue: the task's rows go to xz[out_row + l], zero-padded to RS ----
    T* out = xz + (size_t)task.out_row * RS;
    if constexpr (MODE == 2) {
      // slices summed in slice order through the stage just consumed, QC right-hand sides
      // per round: lane's partial of (its row a, q) at sc[(lane * A2 + a) * QC + q - q0]
      T* sc = reinterpret_cast<T*>(wbase + (size_t)s * warp_stage_bytes((int)sizeof(T)));
      if (task.nunits > 0) {
#pragma unroll
        for (int qc0 = 0; qc0 < R; qc0 += QC) {
          if (js < SL)
#pragma unroll
            for (int a = 0; a < A2; ++a)
#pragma unroll
              for (int qq = 0; qq < QC; ++qq) sc[(lane * A2 + a) * QC + qq] = Ops::get(acc[a], qc0 + qq);
          __syncwarp();
          for (int e = lane; e < O * QC; e += 32) {
            const int row = e / QC, qq = e % QC;
            const int a = (int)(((float)row + 0.5f) * inv);  // row < 128, Og <= 32: exact
            const int l = row - a * Og;
            T v = sc[(l * A2 + a) * QC + qq];
            for (int k = 1; k < SL; ++k) v = v + sc[((k * Og + l) * A2 + a) * QC + qq];
            out[(size_t)row * RS + qc0 + qq] = v;
          }
          __syncwarp();
        }
      } else {
        for (int e = lane; e < O * R; e += 32) out[(size_t)(e / R) * RS + e % R] = zero<T>();
      }
      if constexpr (RS > R)
        for (int e = lane; e < O * (RS - R); e += 32) out[(size_t)(e / (RS - R)) * RS + R + e % (RS - R)] = zero<T>();
    } else {
#pragma unroll
      for (int a = 0; a < A2; ++a) {
        if (a * OL < O) {
          const int l = row0 + a * OL;
          T* row = out + (size_t)l * RS;
#pragma unroll
          for (int q = 0; q < R; ++q) {
            T v = Ops::get(acc[a], q);
            if constexpr (MODE == 1) v = v + shfl_xor(v, 16);
            // MODE 1: half-warp js writes half js of the right-hand sides
            const bool mine = MODE == 0 || (js == 0 ? q < (R + 1) / 2 : q >= (R + 1) / 2);
            if (l < O && mine) row[q] = v;
          }
          if (l < O && js == 0)
#pragma unroll
            for (int q = R; q < RS; ++q) row[q] = zero<T>();
        }
      }
    }
    if (task.nunits > 0 && (kLanes || lane == 0) && (u - 1) + kWarpStages < u_end) {
      // the scratch writes (generic proxy) are ordered before the copy that reuses the stage
      if (lane == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_next(u - 1 + kWarpStages);
    }
    z_chunk_done<T, RS>(task, zred, zcnt, xz, lane);
  }
}

// Warp-level streamed tasks on the tensor cores (FP32 'N' products).  Same per-warp TMA
// pipeline as warp_stream_kernel; the product of a unit is a sequence of warp MMAs
// (mma.sync m16n8k8, TF32 operands, FP32 accumulators) computing out^T = X^T P^T: the
// right-hand sides are the 16 rows of the MMA (A = X^T, one fragment per 8-column step for
// the whole task), the output rows its 8 columns (B = P^T, one fragment per 8-row tile), so an
// output of O rows takes ceil(O / 8) tiles.  FP32 accuracy is kept with the three-term split
// a = a_hi + a_lo (a_hi = a truncated to TF32): X P ~ X_lo P_hi + X_hi P_lo + X_hi P_hi, the
// lo x lo term (2^-20 relative at most) dropped, and every 8-column step goes to fresh
// fragments that are added to the running FP32 sums with round-to-nearest adds (the tensor
// core's own sums are not rounded to nearest).  Operands are read from the stage in fragment
// order (g = lane / 4, t = lane % 4): A holds X[k0 + t (+4)][g (+8)], B holds
// P[k0 + t (+4)][row 8 tile + g]; rows at or past O are computed and never written.  Only the
// last step of a unit whose width is not a multiple of 8 masks its columns (TAIL).
// a_hi = a with its low 13 mantissa bits cleared (a TF32 value), a_lo = a - a_hi (exact in
// FP32; the MMA reads its leading 11 bits).
__device__ __forceinline__ void tf32_split(float v, uint32_t& hi, uint32_t& lo) {
  hi = __float_as_uint(v) & 0xffffe000u;
  lo = __float_as_uint(v - __uint_as_float(hi));
}
// Not volatile: independent tiles' MMA chains may be interleaved by the scheduler.
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One 8-column step k0 of a unit: the A fragment (X^T) once, then the NT 8-row tiles of the
// output (NT a compile-time count, so that the tiles' MMA chains are independent straight-line
// code the scheduler interleaves).  TAIL masks the columns at or past c (both operands: the
// stage past a short piece holds stale data).
template <int RS, int NT, int NTILE, bool TAIL>
__device__ __forceinline__ void mma_kstep(const float* P, const float* X, int k0, int c, int O, int g, int tg,
                                          float (&acc)[NTILE][4]) {
  const int ka = k0 + tg, kb = k0 + tg + 4;
  const bool va = !TAIL || ka < c, vb = !TAIL || kb < c;
  // right-hand sides g and g + 8 of the xz rows (RS columns; the rest are zeros)
  const bool q0 = g < RS, q1 = g + 8 < RS;
  uint32_t ah[4], al[4];
  tf32_split((va && q0) ? X[ka * RS + g] : 0.f, ah[0], al[0]);
  tf32_split((va && q1) ? X[ka * RS + g + 8] : 0.f, ah[1], al[1]);
  tf32_split((vb && q0) ? X[kb * RS + g] : 0.f, ah[2], al[2]);
  tf32_split((vb && q1) ? X[kb * RS + g + 8] : 0.f, ah[3], al[3]);
  const float* pa = P + ka * O + g;
  const float* pb = P + kb * O + g;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    uint32_t bh0, bl0, bh1, bl1;
    tf32_split(va ? pa[t * 8] : 0.f, bh0, bl0);
    tf32_split(vb ? pb[t * 8] : 0.f, bh1, bl1);
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    mma_tf32(d, al, bh0, bh1);
    mma_tf32(d, ah, bl0, bl1);
    mma_tf32(d, ah, bh0, bh1);
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[t][e] += d[e];
  }
}

// All steps of one unit with NT output tiles.
template <int RS, int NT, int NTILE>
__device__ __forceinline__ void mma_unit(const float* P, const float* X, int c, int O, int g, int tg,
                                         float (&acc)[NTILE][4]) {
  int k0 = 0;
  if constexpr (NT <= 4) {
    // two steps per iteration: their MMA chains are independent and overlap (wider tasks
    // have enough independent tiles in one step, and the registers go to their sums; with
    // two steps for 5-7 tiles the y-phase took 0.1213 -> 0.1235 ms, and with them for 4 tiles
    // the z-phase 0.1145 -> 0.111 ms, on the 100,000-point cylinder)
#pragma unroll 2
    for (; k0 + 8 <= c; k0 += 8) mma_kstep<RS, NT, NTILE, false>(P, X, k0, c, O, g, tg, acc);
  } else {
#pragma unroll 1
    for (; k0 + 8 <= c; k0 += 8) mma_kstep<RS, NT, NTILE, false>(P, X, k0, c, O, g, tg, acc);
  }
  if (k0 < c) mma_kstep<RS, NT, NTILE, true>(P, X, k0, c, O, g, tg, acc);
}
// The unit with the task's tile count (1 .. NTILE) as a compile-time constant.
template <typename T, int RS, int NTILE, int NT = 1>
__device__ __forceinline__ void mma_unit_dispatch(int ntn, const T* P, const T* X, int c, int O, int g, int tg,
                                                  T (&acc)[NTILE][4]) {
  if constexpr (NT < NTILE) {
    if (ntn == NT) {
      mma_unit<RS, NT, NTILE>(P, X, c, O, g, tg, acc);
      return;
    }
    mma_unit_dispatch<T, RS, NTILE, NT + 1>(ntn, P, X, c, O, g, tg, acc);
  } else {
    mma_unit<RS, NTILE, NTILE>(P, X, c, O, g, tg, acc);
  }
}

// CTAs an SM the tensor-core kernel is compiled for: four, the number its shared memory allows
// (two stages of warp_stage_bytes(4) for each of its four warps), so every tile count gets the
// registers of four CTAs.
__host__ __device__ constexpr int mma_min_blocks(int /*ntile*/, int /*elem_bytes*/) { return 4; }

template <typename T, int R, int RS, int NTILE>
__global__ void __launch_bounds__(kWarpCTA * 32, mma_min_blocks(NTILE, sizeof(T)))
    mma_stream_kernel(const GemvTask* __restrict__ tasks, const int* __restrict__ warp_begin,
                      const GemvUnit* __restrict__ units, const T* __restrict__ arena, T* xz, GemvStatus* err,
                      const GemvZred* __restrict__ zred, int* zcnt) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  pdl_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tg = lane & 3;
  unsigned char* wbase = smem_raw + (size_t)warp * kWarpStages * warp_stage_bytes((int)sizeof(T));
  // per stage: the unit's column count and X offset (what the consumers read), then the barriers
  int2* uslot =
      reinterpret_cast<int2*>(smem_raw + (size_t)kWarpCTA * kWarpStages * warp_stage_bytes((int)sizeof(T))) + warp * kWarpStages;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kWarpCTA * kWarpStages *
                                                               (warp_stage_bytes((int)sizeof(T)) + sizeof(int2))) +
                   warp * kWarpStages;
  const int gw = blockIdx.x * kWarpCTA + warp;
  const int t0 = warp_begin[gw], t1 = warp_begin[gw + 1];
  if (t0 >= t1) return;
  const int u_begin = tasks[t0].first_unit;
  const int u_end = tasks[t1 - 1].first_unit + tasks[t1 - 1].nunits;
  const long long wlim = err->wait_limit;

  if (lane == 0) {
    for (int s = 0; s < kWarpStages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncwarp();
  constexpr bool kLanes = NTILE <= 8;  // descriptors spread over the lanes (NextUnit)
  NextUnit<kLanes> nxt;
  int last_issued = u_begin - 1;  // lane 0: the last unit whose copies were issued
  auto issue = [&](int u, const GemvUnit& U) {
    const int s = (u - u_begin) % kWarpStages;
    last_issued = u;
    uslot[s] = make_int2(U.c, U.o0);
    const uint32_t pbytes = round16((uint64_t)U.pel * sizeof(T));
    const uint32_t xbytes = (uint32_t)U.c * RS * (uint32_t)sizeof(T);
    unsigned char* st = wbase + (size_t)s * warp_stage_bytes((int)sizeof(T));
    if (!unit_copies_ok<T, RS>(U, arena, xz, warp_stage_bytes((int)sizeof(T)), U.o0)) {
      record_bad_unit(err, u);
      mbar_arrive(&bars[s]);
      return;
    }
    mbar_expect_tx(&bars[s], pbytes + xbytes);
    bulk_piece(st, arena + U.poff, pbytes, &bars[s]);
    issue_x<T, RS>(st + U.o0, xz, U, &bars[s]);
  };
  auto issue_next = [&](int v) {  // nxt holds units[v]; kLanes: every lane calls it, else lane 0
    const GemvUnit U = nxt.get();
    if (lane == 0) issue(v, U);
    if (v + 1 < u_end) nxt.load(units, v + 1, lane);
  };
  if (lane == 0)
    for (int v = u_begin; v < u_end && v < u_begin + kWarpStages; ++v) issue(v, units[v]);
  if (u_begin + kWarpStages < u_end) nxt.load(units, u_begin + kWarpStages, lane);

  int u = u_begin;
  NextTask<kLanes> task_next;
  task_next.load(tasks, t0, lane);
  for (int t = t0; t < t1; ++t) {
    const GemvTask task = task_next.get();
    if (t + 1 < t1) task_next.load(tasks, t + 1, lane);
    const int O = task.O;
    const int ntn = (O + 7) >> 3;  // 8-row tiles holding rows of this task (warp-uniform)
    T acc[NTILE][4];
#pragma unroll
    for (int i = 0; i < NTILE; ++i)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][e] = zero<T>();

    for (int kk = 0; kk < task.nunits; ++kk, ++u) {
      const int s = (u - u_begin) % kWarpStages;
      const uint32_t parity = (uint32_t)(((u - u_begin) / kWarpStages) & 1);
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[s], parity, wlim))) {
        if (lane == 0) warp_give_up(err, bars, kWarpStages, u_begin, u, last_issued);
        return;
      }
      const int c = uslot[s].x;
      const T* P = reinterpret_cast<const T*>(wbase + (size_t)s * warp_stage_bytes((int)sizeof(T)));
      const T* X = reinterpret_cast<const T*>(wbase + (size_t)s * warp_stage_bytes((int)sizeof(T)) + uslot[s].y);
      mma_unit_dispatch<T, RS, NTILE>(ntn, P, X, c, O, g, tg, acc);
      __syncwarp();  // every lane is done with stage s
      if ((kLanes || lane == 0) && u + kWarpStages < u_end) issue_next(u + kWarpStages);
    }

    // ---- epilogue: accumulator (rhs g (+8), rows 8 i + 2 t (+1)); right-hand sides past R
    // hold exact zeros (their X columns were zeros), which pads the row to RS ----
    T* out = xz + (size_t)task.out_row * RS;
#pragma unroll
    for (int i = 0; i < NTILE; ++i) {
      if (i < ntn) {
        const int r0 = i * 8 + 2 * tg, r1 = r0 + 1;
        if (g < RS) {
          if (r0 < O) out[(size_t)r0 * RS + g] = acc[i][0];
          if (r1 < O) out[(size_t)r1 * RS + g] = acc[i][1];
        }
        if (g + 8 < RS) {
          if (r0 < O) out[(size_t)r0 * RS + g + 8] = acc[i][2];
          if (r1 < O) out[(size_t)r1 * RS + g + 8] = acc[i][3];
        }
      }
    }
    z_chunk_done<T, RS>(task, zred, zcnt, xz, lane);
  }
}

// ---------------------------------------------------------------------------------
// FP32 'N' product on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor
// memory), one task at a time per CTA of 128 threads; thread t owns output row t.
//
// A unit out(O x 16) += P (O x c) X (c x 16), c <= kTcCols, is D = A B^T with A = P
// (M = 128, K = c) and B = X^T (N = 16, K = c): TF32 operands in shared memory, K-major
// without swizzle (8-row x 16-byte core matrices, 128 B between the two 4-column halves of a
// k-step, 256 B between 8-row groups).  FP32 accuracy as in the warp-level kernel: the split
// P X ~ P_lo X_hi + P_hi X_lo + P_hi X_hi, each 8-column step into its own accumulator
// (tensor-memory columns 16 s) and the steps added in order to the running sums in registers
// with FP32 round-to-nearest adds (the tensor core's own sums are not rounded to nearest).
// Thread 0 streams the pieces through a ring of kTcStages stages (cp.async.bulk + mbarrier),
// issues the MMAs and commits them to an mbarrier; all threads split the raw piece into the
// hi / lo tiles and read the accumulators back (tcgen05.ld, one 32-lane quarter per warp).
// Tile rows at or past O are not written: they hold what earlier units left and only reach
// output rows that are never stored.  Every wait is bounded and sets `err` when it gives up.
constexpr int kTcThreads = 128;
constexpr int kTcStages = 4;
constexpr int kTcSteps = kTcCols / 8;
constexpr int kTcTileA = 128 * 8 * 4;  // one k-step of A: 4 KB
constexpr int kTcTileB = 16 * 8 * 4;   // one k-step of B: 512 B
constexpr int kTcStage = kTcPieceBytes + kTcXBytes;
constexpr int kTcTmemCols = 16 * kTcSteps;  // a power of two >= 32
constexpr uint32_t kTcIdesc = (1u << 4)     // D: F32
                              | (2u << 7)   // A: TF32
                              | (2u << 10)  // B: TF32
                              | (2u << 17)  // N = 16
                              | (8u << 24); // M = 128

__device__ __forceinline__ uint32_t tc_kmaj(int r, int k) {
  return (uint32_t)((r >> 3) * 256 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ uint64_t tc_desc(const void* p) {
  const uint32_t a = smem_u32(p);
  return (uint64_t)((a >> 4) & 0x3fff) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
         ((uint64_t)1 << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate));
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&f)[16]) {
  uint32_t v[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(v[i]);
}
__device__ __forceinline__ float4 tc_hi(float4 v, float4& lo) {
  float4 h;
  h.x = __uint_as_float(__float_as_uint(v.x) & 0xffffe000u);
  h.y = __uint_as_float(__float_as_uint(v.y) & 0xffffe000u);
  h.z = __uint_as_float(__float_as_uint(v.z) & 0xffffe000u);
  h.w = __uint_as_float(__float_as_uint(v.w) & 0xffffe000u);
  lo = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
  return h;
}

template <int RS>
__global__ void __launch_bounds__(kTcThreads, 1)
    umma_stream_kernel(const GemvTask* __restrict__ tasks, const int* __restrict__ cta_begin,
                       const GemvUnit* __restrict__ units, const float* __restrict__ arena, float* xz, GemvStatus* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* ring = smem_raw;
  unsigned char* tAh = ring + kTcStages * kTcStage;
  unsigned char* tAl = tAh + kTcSteps * kTcTileA;
  unsigned char* tBh = tAl + kTcSteps * kTcTileA;
  unsigned char* tBl = tBh + kTcSteps * kTcTileB;
  uint64_t* full = reinterpret_cast<uint64_t*>(tBl + kTcSteps * kTcTileB);
  uint64_t* mmab = full + kTcStages;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mmab + 1);
  GemvUnit* uslot = reinterpret_cast<GemvUnit*>(tslot + 4);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int t0 = cta_begin[blockIdx.x], t1 = cta_begin[blockIdx.x + 1];
  if (t0 >= t1) return;
  const int u_begin = tasks[t0].first_unit;
  const int u_end = tasks[t1 - 1].first_unit + tasks[t1 - 1].nunits;
  const long long wlim = err->wait_limit;
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) mbar_init(&full[s], 1);
    mbar_init(mmab, 1);
    mbar_fence_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);

  int last_issued = u_begin - 1;  // thread 0: the last unit whose copies were issued
  auto issue = [&](int v) {
    const GemvUnit U = units[v];
    const int s = (v - u_begin) % kTcStages;
    last_issued = v;
    uslot[s] = U;
    const uint32_t pbytes = round16((uint64_t)U.pel * sizeof(float));
    const uint32_t xbytes = (uint32_t)U.c * RS * (uint32_t)sizeof(float);
    unsigned char* st = ring + (size_t)s * kTcStage;
    mbar_expect_tx(&full[s], pbytes + xbytes);
    bulk_piece(st, arena + U.poff, pbytes, &full[s]);
    issue_x<float, RS>(st + kTcPieceBytes, xz, U, &full[s]);
  };
  if (tid == 0)
    for (int v = u_begin; v < u_end && v < u_begin + kTcStages; ++v) issue(v);

  uint32_t mma_parity = 0;
  int u = u_begin;
  // a wait that gives up stops the CTA (CTA-uniform): `pending` is the first unit whose
  // copies are not consumed, `mma_pending` whether a commit is not waited for
  bool failed = false, mma_pending = false;
  int pending = u_begin;
  for (int t = t0; t < t1 && !failed; ++t) {
    const GemvTask task = tasks[t];
    const int O = task.O;
    float acc[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) acc[n] = 0.f;
    for (int kk = 0; kk < task.nunits; ++kk, ++u) {
      const int s = (u - u_begin) % kTcStages;
      if (__syncthreads_or(!mbar_wait_bounded(&full[s], (uint32_t)(((u - u_begin) / kTcStages) & 1), wlim))) {
        failed = true;
        pending = u;
        break;
      }
      const int c = uslot[s].c;
      const float* P = reinterpret_cast<const float*>(ring + (size_t)s * kTcStage);
      const float* X = reinterpret_cast<const float*>(ring + (size_t)s * kTcStage + kTcPieceBytes);
      // A tiles: (row i, 4-column quad q), rows < O, columns past c as zeros
      for (int it = tid; it < O * (kTcCols / 4); it += kTcThreads) {
        const int i = it % O, q = it / O, k0 = 4 * q;
        float4 v;
        v.x = k0 < c ? P[(size_t)k0 * O + i] : 0.f;
        v.y = k0 + 1 < c ? P[(size_t)(k0 + 1) * O + i] : 0.f;
        v.z = k0 + 2 < c ? P[(size_t)(k0 + 2) * O + i] : 0.f;
        v.w = k0 + 3 < c ? P[(size_t)(k0 + 3) * O + i] : 0.f;
        float4 lo;
        const float4 hi = tc_hi(v, lo);
        const uint32_t off = (uint32_t)(q >> 1) * kTcTileA + tc_kmaj(i, (q & 1) * 4);
        *reinterpret_cast<float4*>(tAh + off) = hi;
        *reinterpret_cast<float4*>(tAl + off) = lo;
      }
      // B tiles: (right-hand side n, quad q), exactly one item a thread
      {
        const int n = tid & 15, q = tid >> 4, k0 = 4 * q;
        float4 v;
        v.x = (n < RS && k0 < c) ? X[(size_t)k0 * RS + n] : 0.f;
        v.y = (n < RS && k0 + 1 < c) ? X[(size_t)(k0 + 1) * RS + n] : 0.f;
        v.z = (n < RS && k0 + 2 < c) ? X[(size_t)(k0 + 2) * RS + n] : 0.f;
        v.w = (n < RS && k0 + 3 < c) ? X[(size_t)(k0 + 3) * RS + n] : 0.f;
        float4 lo;
        const float4 hi = tc_hi(v, lo);
        const uint32_t off = (uint32_t)(q >> 1) * kTcTileB + tc_kmaj(n, (q & 1) * 4);
        *reinterpret_cast<float4*>(tBh + off) = hi;
        *reinterpret_cast<float4*>(tBl + off) = lo;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();  // tiles written, stage s read
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int nsteps = (c + 7) >> 3;
      if (tid == 0) {
        for (int st = 0; st < nsteps; ++st) {
          const uint64_t ah = tc_desc(tAh + st * kTcTileA), al = tc_desc(tAl + st * kTcTileA);
          const uint64_t bh = tc_desc(tBh + st * kTcTileB), bl = tc_desc(tBl + st * kTcTileB);
          const uint32_t d = tmem + 16 * st;
          tc_mma(d, al, bh, 0);
          tc_mma(d, ah, bl, 1);
          tc_mma(d, ah, bh, 1);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(mmab))
                     : "memory");
        if (u + kTcStages < u_end) issue(u + kTcStages);
      }
      if (__syncthreads_or(!mbar_wait_bounded(mmab, mma_parity, wlim))) {
        failed = mma_pending = true;
        pending = u + 1;
        break;
      }
      mma_parity ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int st = 0; st < nsteps; ++st) {
        float f[16];
        tc_ld16(tlane + 16 * st, f);
#pragma unroll
        for (int n = 0; n < 16; ++n) acc[n] = __fadd_rn(acc[n], f[n]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (failed) break;
    if (tid < O) {
      float* out = xz + (size_t)(task.out_row + tid) * RS;
      if constexpr (RS % 4 == 0) {
#pragma unroll
        for (int n = 0; n < RS; n += 4)
          *reinterpret_cast<float4*>(out + n) = make_float4(acc[n], acc[n + 1], acc[n + 2], acc[n + 3]);
      } else {
#pragma unroll
        for (int n = 0; n < RS; ++n) out[n] = acc[n];
      }
    }
  }
  if (failed && tid == 0) {
    // flag the product, then let the MMAs and copies in flight finish before the tensor
    // memory is freed and the CTA exits
    atomicExch(&err->failed, 1);
    if (mma_pending) mbar_wait_bounded(mmab, mma_parity, drain_limit(err));
    for (int v = pending; v <= last_issued; ++v)
      mbar_wait_bounded(&full[(v - u_begin) % kTcStages], (uint32_t)(((v - u_begin) / kTcStages) & 1),
                        drain_limit(err));
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
}

template <int RS>
void launch_umma_t(const GemvLaunch& L, const GemvUnit* units, const float* arena, float* xz, GemvStatus* err,
                   cudaStream_t s) {
  auto kern = umma_stream_kernel<RS>;
  const size_t smem = (size_t)kTcStages * kTcStage + 2 * kTcSteps * (kTcTileA + kTcTileB) + (kTcStages + 1) * 8 +
                      16 + kTcStages * sizeof(GemvUnit);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  kern<<<L.ncta, kTcThreads, smem, s>>>(L.tasks, L.cta_begin, units, arena, xz, err);
}

// y in client order from the partial rows of the 'N' y tasks:
// y[i, q0 + q] = alpha * sum_p xz[pos + p * O, q] + beta * y[i, q0 + q].  A CTA takes 128
// client rows: the partial rows are read along q (contiguous), transposed through shared
// memory, and y is written along i (contiguous in each column of y).
constexpr int kFinalRows = 128;
template <typename T, int R, int RS>
__global__ void __launch_bounds__(256) yfinal_kernel(const int2* __restrict__ rows, int n, const T* __restrict__ xz,
                                                     T* __restrict__ y, int ldy, int q0, int r, T alpha, T beta) {
  __shared__ T tile[R][kFinalRows + 1];
  __shared__ int2 rd[kFinalRows];
  pdl_wait();
  const int i0 = blockIdx.x * kFinalRows;
  // the rows' part descriptors first, so that the loads of the partial rows below do not wait
  // on them one by one
  for (int il = threadIdx.x; il < kFinalRows; il += blockDim.x) rd[il] = i0 + il < n ? rows[i0 + il] : int2{0, 0};
  __syncthreads();
#pragma unroll 4
  for (int e = threadIdx.x; e < kFinalRows * R; e += blockDim.x) {
    const int il = e / R, q = e % R;
    const int2 d = rd[il];
    const int O = d.y & 255, np = d.y >> 8;
    T v = zero<T>();
    for (int p = 0; p < np; ++p) v = v + xz[((size_t)d.x + (size_t)p * O) * RS + q];
    tile[q][il] = v;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kFinalRows * R; e += blockDim.x) {
    const int q = e / kFinalRows, il = e % kFinalRows, i = i0 + il;
    if (i < n && q0 + q < r) {
      T* yp = y + (size_t)i + (size_t)(q0 + q) * ldy;
      T outv = alpha * tile[q][il];
      if (!is_zero_val(beta)) outv = fmadd(beta, *yp, outv);
      *yp = outv;
    }
  }
}

// Sums the chunk partials of long leaves: xz[final + l] = sum_p xz[part + p k + l], the parts
// added in part order.  A warp per sum (kZredWarps sums a CTA), lanes over 16-byte chunks of
// the k x RS slot (a row of RS scalars is a multiple of 16 bytes).
constexpr int kZredWarps = 8;
template <typename T, int RS>
__global__ void __launch_bounds__(kZredWarps * 32) zred_kernel(const GemvZred* __restrict__ zr, int n, T* xz) {
  constexpr int V = sizeof(T) >= 16 ? 1 : 16 / (int)sizeof(T);  // scalars a 16-byte chunk
  static_assert((RS * sizeof(T)) % 16 == 0, "xz rows are 16-byte multiples");
  pdl_wait();
  const int w = blockIdx.x * kZredWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (w >= n) return;
  const GemvZred d = zr[w];
  const int nchunk = d.k * RS / V;
  const T* part = xz + (size_t)d.part_row * RS;
  T* fin = xz + (size_t)d.final_row * RS;
  constexpr int kBatch = 8;  // parts loaded before they are added (loads in flight together)
  for (int c = lane; c < nchunk; c += 32) {
    T s[V];
#pragma unroll
    for (int e = 0; e < V; ++e) s[e] = zero<T>();
    for (int p0 = 0; p0 < d.nparts; p0 += kBatch) {
      uint4 raw[kBatch];
#pragma unroll
      for (int i = 0; i < kBatch; ++i)
        if (p0 + i < d.nparts)
          raw[i] = *reinterpret_cast<const uint4*>(part + ((size_t)(p0 + i) * d.k * RS + (size_t)c * V));
#pragma unroll
      for (int i = 0; i < kBatch; ++i)
        if (p0 + i < d.nparts) {
          const T* v = reinterpret_cast<const T*>(&raw[i]);
#pragma unroll
          for (int e = 0; e < V; ++e) s[e] = s[e] + v[e];
        }
    }
    *reinterpret_cast<uint4*>(fin + (size_t)c * V) = *reinterpret_cast<const uint4*>(s);
  }
}
inline unsigned zred_grid(int n) { return (unsigned)((n + kZredWarps - 1) / kZredWarps); }

// A launch with programmatic stream serialization (see pdl_wait): the kernel must begin with
// pdl_wait() before it reads what the kernel before it wrote.
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, args...);  // errors surface through cudaGetLastError, as for <<<>>>
}

// ---------------------------------------------------------------------------------
template <typename T, int R, int RS, int OL, int RPT, bool TRANSP>
void launch_stream_t(const GemvLaunch& L, const GemvUnit* units, const T* arena, T* xz, int conj,
                     const int* perm_out, T* y, int ldy, int q0, int r, T alpha, T beta, GemvStatus* err, cudaStream_t s) {
  constexpr int NSTAGE = nstage_of<T>();
  auto kern = stream_kernel<T, R, RS, OL, RPT, TRANSP, NSTAGE>;
  const size_t smem = stream_smem_bytes(sizeof(T), R, RS, OL * RPT, TRANSP);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  kern<<<L.ncta, kThreads, smem, s>>>(L.tasks, L.cta_begin, units, arena, xz, conj, L.out_is_y ? 1 : 0, perm_out, y,
                                       ldy, q0, r, alpha, beta, err);
}

template <typename T, int R, int RS, int MODE, int A2>
void launch_warp_t(const GemvLaunch& L, const GemvUnit* units, const T* arena, T* xz, GemvStatus* err, cudaStream_t s,
                   const GemvZred* zred, int* zcnt) {
  auto kern = warp_stream_kernel<T, R, RS, MODE, A2>;
  const size_t smem = warp_stream_smem_bytes((int)sizeof(T));
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  launch_pdl(kern, dim3(L.ncta), dim3(kWarpCTA * 32), smem, s, L.tasks, L.cta_begin, units, arena, xz, err, zred,
             zcnt);
}

template <typename T, int R, int RS, int NTILE>
void launch_mma_t(const GemvLaunch& L, const GemvUnit* units, const T* arena, T* xz, GemvStatus* err,
                  cudaStream_t s, const GemvZred* zred, int* zcnt) {
  auto kern = mma_stream_kernel<T, R, RS, NTILE>;
  const size_t smem = warp_stream_smem_bytes((int)sizeof(T));
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  launch_pdl(kern, dim3(L.ncta), dim3(kWarpCTA * 32), smem, s, L.tasks, L.cta_begin, units, arena, xz, err, zred,
             zcnt);
}

// zred / zcnt: the sums of the z chunks, done by the warp-level z kernels themselves
// (z_chunk_done); null for the y launches and the CTA-level kernels.
template <typename T, int R, int RS, bool TRANSP>
void launch_stream(const GemvLaunch& L, const GemvUnit* units, const T* arena, T* xz, int conj, const int* perm_out,
                   T* y, int ldy, int q0, int r, T alpha, T beta, GemvStatus* err, cudaStream_t s,
                   const GemvZred* zred = nullptr, int* zcnt = nullptr) {
  if (L.ntasks <= 0) return;
  if constexpr (std::is_same<T, float>::value && !TRANSP) {
    if (L.map == 4) {
      launch_umma_t<RS>(L, units, arena, xz, err, s);
      return;
    }
  }
  if (L.warp_level) {
    if constexpr (std::is_same<T, float>::value) {
      if (L.map == 3) {  // rpt = 8-row tiles of the launch's tallest task (exact up to 8)
        switch (L.rpt) {
          case 1: launch_mma_t<T, R, RS, 1>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 2: launch_mma_t<T, R, RS, 2>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 3: launch_mma_t<T, R, RS, 3>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 4: launch_mma_t<T, R, RS, 4>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 5: launch_mma_t<T, R, RS, 5>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 6: launch_mma_t<T, R, RS, 6>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 7: launch_mma_t<T, R, RS, 7>(L, units, arena, xz, err, s, zred, zcnt); break;
          case 8: launch_mma_t<T, R, RS, 8>(L, units, arena, xz, err, s, zred, zcnt); break;
          default: launch_mma_t<T, R, RS, 16>(L, units, arena, xz, err, s, zred, zcnt); break;
        }
        return;
      }
    }
    if (L.map == 2)
      launch_warp_t<T, R, RS, 2, 2>(L, units, arena, xz, err, s, zred, zcnt);
    else if (L.map == 5)
      launch_warp_t<T, R, RS, 0, 2>(L, units, arena, xz, err, s, zred, zcnt);
    else if (L.map == 1)
      launch_warp_t<T, R, RS, 1, 4>(L, units, arena, xz, err, s, zred, zcnt);
    else
      launch_warp_t<T, R, RS, 0, 4>(L, units, arena, xz, err, s, zred, zcnt);
    return;
  }
  if (L.ol == 16)
    launch_stream_t<T, R, RS, 16, 1, TRANSP>(L, units, arena, xz, conj, perm_out, y, ldy, q0, r, alpha, beta, err, s);
  else if (L.rpt == 1)
    launch_stream_t<T, R, RS, 32, 1, TRANSP>(L, units, arena, xz, conj, perm_out, y, ldy, q0, r, alpha, beta, err, s);
  else if (L.rpt == 2)
    launch_stream_t<T, R, RS, 32, 2, TRANSP>(L, units, arena, xz, conj, perm_out, y, ldy, q0, r, alpha, beta, err, s);
  else
    launch_stream_t<T, R, RS, 32, 4, TRANSP>(L, units, arena, xz, conj, perm_out, y, ldy, q0, r, alpha, beta, err, s);
}

template <typename T, int R, bool TRANSP>
void run_tile(const GemvPlan& p, int nrhs, int q0, T alpha, T beta, const T* x, T* y, T* xz, int conj, GemvStatus* err,
              cudaStream_t s, const GemvTiming* tm) {
  constexpr int RS = rs_of<T>(R);
  const GemvSide& side = p.side[TRANSP ? 1 : 0];
  const int n_in = TRANSP ? p.n_rows : p.n_cols;
  const int* iperm_in = TRANSP ? p.iperm_rows : p.iperm_cols;
  const int* perm_out = TRANSP ? p.perm_cols : p.perm_rows;
  const int ld_in = n_in, ld_out = TRANSP ? p.n_cols : p.n_rows;
  const T* arena = (const T*)p.arena;
  if (tm) cudaEventRecord(tm->ev[0], s);
  const GemvSide& sn = p.side[0];
  gather_kernel<T, R, RS><<<gather_grid(n_in), 256, 0, s>>>(x, n_in, ld_in, q0, nrhs, iperm_in, xz, p.n_in_max, sn.zcnt,
                                                            sn.zfused ? sn.nzred : 0);
  if (tm) cudaEventRecord(tm->ev[1], s);
  for (int c = 0; c < side.nz; ++c)
    launch_stream<T, R, RS, TRANSP>(side.z[c], side.units, arena, xz, conj, nullptr, nullptr, 0, 0, 0, alpha, beta,
                                    err, s, side.zfused ? side.zred : nullptr, side.zcnt);
  if (side.nzred > 0 && !side.zfused) launch_pdl(zred_kernel<T, RS>, dim3(zred_grid(side.nzred)), dim3(kZredWarps * 32), 0, s, side.zred, side.nzred, xz);
  if (tm) cudaEventRecord(tm->ev[2], s);
  launch_stream<T, R, RS, TRANSP>(side.y, side.units, arena, xz, conj, perm_out, y, ld_out, q0, nrhs, alpha, beta,
                                  err, s);
  if (side.nyrows > 0) {
    const unsigned nb = (unsigned)((side.nyrows + kFinalRows - 1) / kFinalRows);
    launch_pdl(yfinal_kernel<T, R, RS>, dim3(nb), dim3(256), 0, s, side.yrows, side.nyrows, xz, y, ld_out, q0, nrhs,
               alpha, beta);
  }
  if (tm) cudaEventRecord(tm->ev[3], s);
}

template <typename T, bool TRANSP>
void run_all(const GemvPlan& p, int nrhs, T alpha, T beta, const T* x, T* y, T* xz, int conj, GemvStatus* err,
             cudaStream_t s, const GemvTiming* tm) {
  // complex double keeps tiles of at most 4 right-hand sides (shared-memory budget)
  constexpr int maxR = sizeof(T) >= 16 ? 4 : 16;
  for (int q0 = 0; q0 < nrhs; q0 += maxR) {
    const int rem = nrhs - q0;
    if (maxR == 16 && rem > 8) run_tile<T, (maxR >= 16 ? 16 : 4), TRANSP>(p, nrhs, q0, alpha, beta, x, y, xz, conj, err, s, tm);
    else if (maxR == 16 && rem > 4) run_tile<T, (maxR >= 16 ? 8 : 4), TRANSP>(p, nrhs, q0, alpha, beta, x, y, xz, conj, err, s, tm);
    else if (rem > 1) run_tile<T, 4, TRANSP>(p, nrhs, q0, alpha, beta, x, y, xz, conj, err, s, tm);
    else run_tile<T, 1, TRANSP>(p, nrhs, q0, alpha, beta, x, y, xz, conj, err, s, tm);
  }
}

// ---------------------------------------------------------------------------------
// Leaf-factor gradients (adjoint of y = H x with respect to the stored leaves), written in
// the canonical layout (full: m x n, Rk: A m x k then B n x k, column-major).
// R is the right-hand-side tile (compile time): columns past the caller's count hold exact
// zeros in xs and rs (the gather pads them), so they add nothing.
template <typename T, int RS, int R>
__global__ void grad_full_kernel(const GemvFullLeaf* __restrict__ full, int nfull, const T* __restrict__ xs,
                                 const T* __restrict__ rs, T* __restrict__ g, bool accumulate) {
  // warp per column j of a leaf, lanes over its rows: coalesced column writes, no division
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int f = blockIdx.x; f < nfull; f += gridDim.x) {
    const GemvFullLeaf F = full[f];
    for (int j = warp; j < F.n; j += nw) {
      const T* xv = xs + (size_t)(F.col_off + j) * RS;
      T* dF = g + F.goff + (size_t)j * F.m;
      for (int i = lane; i < F.m; i += 32) {
        const T* rv = rs + (size_t)(F.row_off + i) * RS;
        T acc = accumulate ? dF[i] : zero<T>();
#pragma unroll
        for (int q = 0; q < R; ++q) acc = fmadd(rv[q], xv[q], acc);
        dF[i] = acc;
      }
    }
  }
}

template <typename T, int RS, int R>
__global__ void grad_rk_kernel(const GemvRkLeaf* __restrict__ rk, int nrk, const T* __restrict__ xs,
                               const T* __restrict__ rs, T* __restrict__ g, bool accumulate) {
  // warp per factor column l, lanes over rows: coalesced column writes, no division
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = blockIdx.x; t < nrk; t += gridDim.x) {
    const GemvRkLeaf L = rk[t];
    T* dA = g + L.goff;
    T* dB = dA + (size_t)L.m * L.k;
    // dA[i, l] = sum_q r[i, q] z[l, q],  z = B^T x  (rows zrow_n of the x buffer)
    for (int l = warp; l < L.k; l += nw) {
      const T* zv = xs + (size_t)(L.zrow_n + l) * RS;
      T* col = dA + (size_t)l * L.m;
      for (int i = lane; i < L.m; i += 32) {
        const T* rv = rs + (size_t)(L.row_off + i) * RS;
        T acc = accumulate ? col[i] : zero<T>();
#pragma unroll
        for (int q = 0; q < R; ++q) acc = fmadd(rv[q], zv[q], acc);
        col[i] = acc;
      }
    }
    // dB[j, l] = sum_q x[j, q] w[l, q],  w = A^T r  (rows zrow_t of the r buffer)
    for (int l = warp; l < L.k; l += nw) {
      const T* wv = rs + (size_t)(L.zrow_t + l) * RS;
      T* col = dB + (size_t)l * L.n;
      for (int j = lane; j < L.n; j += 32) {
        const T* xv = xs + (size_t)(L.col_off + j) * RS;
        T acc = accumulate ? col[j] : zero<T>();
#pragma unroll
        for (int q = 0; q < R; ++q) acc = fmadd(xv[q], wv[q], acc);
        col[j] = acc;
      }
    }
  }
}

template <typename T, int R>
void grads_tile(const GemvPlan& p, int nrhs, const T* x, const T* r, T* xz, T* rz, T* gfull, T* grk, bool accumulate,
                GemvStatus* err, cudaStream_t s) {
  constexpr int RS = rs_of<T>(R);
  const T* arena = (const T*)p.arena;
  // x in cluster order (columns) and z = B^T x
  const GemvSide& sn = p.side[0];
  gather_kernel<T, R, RS><<<gather_grid(p.n_cols), 256, 0, s>>>(x, p.n_cols, p.n_cols, 0, nrhs, p.iperm_cols, xz,
                                                                   p.n_in_max, sn.zcnt, sn.zfused ? sn.nzred : 0);
  for (int c = 0; c < sn.nz; ++c)
    launch_stream<T, R, RS, false>(sn.z[c], sn.units, arena, xz, 0, nullptr, nullptr, 0, 0, 0, one<T>(), zero<T>(),
                                   err, s, sn.zfused ? sn.zred : nullptr, sn.zcnt);
  if (sn.nzred > 0 && !sn.zfused) launch_pdl(zred_kernel<T, RS>, dim3(zred_grid(sn.nzred)), dim3(kZredWarps * 32), 0, s, sn.zred, sn.nzred, xz);
  // r in cluster order (rows) and w = A^T r
  gather_kernel<T, R, RS><<<gather_grid(p.n_rows), 256, 0, s>>>(r, p.n_rows, p.n_rows, 0, nrhs, p.iperm_rows, rz,
                                                                   p.n_in_max, sn.zcnt, sn.zfused ? sn.nzred : 0);
  const GemvSide& st = p.side[1];
  for (int c = 0; c < st.nz; ++c)
    launch_stream<T, R, RS, true>(st.z[c], st.units, arena, rz, 0, nullptr, nullptr, 0, 0, 0, one<T>(), zero<T>(),
                                  err, s);
  if (st.nzred > 0) launch_pdl(zred_kernel<T, RS>, dim3(zred_grid(st.nzred)), dim3(kZredWarps * 32), 0, s, st.zred, st.nzred, rz);
  const int grid = persistent_grid(4);
  if (p.nfull > 0 && gfull)
    grad_full_kernel<T, RS, R><<<grid, 256, 0, s>>>(p.full, p.nfull, xz, rz, gfull, accumulate);
  if (p.nrk > 0 && grk) grad_rk_kernel<T, RS, R><<<grid, 256, 0, s>>>(p.rk, p.nrk, xz, rz, grk, accumulate);
}

// The adjoint of y = H x at the output gradient r in one pass: dx = H^T r (the 'T' product,
// whose z' = A^T r stays in rz) and the leaf gradients, which reuse that z' as w; z = B^T x is
// formed once in xz.
template <typename T, int R>
void adjoint_tile(const GemvPlan& p, int nrhs, const T* x, const T* r, T* dx, T* xz, T* rz, T* gfull, T* grk,
                  bool accumulate, GemvStatus* err, cudaStream_t s) {
  constexpr int RS = rs_of<T>(R);
  const T* arena = (const T*)p.arena;
  run_tile<T, R, true>(p, nrhs, 0, one<T>(), zero<T>(), r, dx, rz, 0, err, s, nullptr);
  const GemvSide& sn = p.side[0];
  gather_kernel<T, R, RS><<<gather_grid(p.n_cols), 256, 0, s>>>(x, p.n_cols, p.n_cols, 0, nrhs, p.iperm_cols, xz,
                                                                   p.n_in_max, sn.zcnt, sn.zfused ? sn.nzred : 0);
  for (int c = 0; c < sn.nz; ++c)
    launch_stream<T, R, RS, false>(sn.z[c], sn.units, arena, xz, 0, nullptr, nullptr, 0, 0, 0, one<T>(), zero<T>(),
                                   err, s, sn.zfused ? sn.zred : nullptr, sn.zcnt);
  if (sn.nzred > 0 && !sn.zfused) launch_pdl(zred_kernel<T, RS>, dim3(zred_grid(sn.nzred)), dim3(kZredWarps * 32), 0, s, sn.zred, sn.nzred, xz);
  const int grid = persistent_grid(4);
  if (p.nfull > 0 && gfull)
    grad_full_kernel<T, RS, R><<<grid, 256, 0, s>>>(p.full, p.nfull, xz, rz, gfull, accumulate);
  if (p.nrk > 0 && grk) grad_rk_kernel<T, RS, R><<<grid, 256, 0, s>>>(p.rk, p.nrk, xz, rz, grk, accumulate);
}

}  // namespace

size_t stream_smem_bytes(int elem_bytes, int R, int RS, int omax, bool transposed) {
  const int nstage = elem_bytes >= 16 ? 2 : 3;
  const size_t xcap = (size_t)(transposed ? kMaxInner : kPieceCols) * RS;
  const size_t pcap = (size_t)kPieceElems + 2 * omax + 16;
  return (size_t)nstage * (pcap + xcap) * elem_bytes + (size_t)kWarps * omax * R * elem_bytes + nstage * 8 + 16;
}

int gemv_rhs_stride(int elem_bytes, int R) { return R * elem_bytes >= 16 ? R : 16 / elem_bytes; }

size_t warp_stream_smem_bytes(int elem_bytes) {
  return (size_t)kWarpCTA * kWarpStages * (warp_stage_bytes(elem_bytes) + sizeof(int2) + sizeof(uint64_t));
}
int warp_stream_warps_per_cta() { return kWarpCTA; }
int mma_stream_blocks_per_sm(int ntile, int elem_bytes) { return mma_min_blocks(ntile, elem_bytes); }

size_t umma_smem_bytes() {
  return (size_t)kTcStages * kTcStage + 2 * kTcSteps * (kTcTileA + kTcTileB) + (kTcStages + 1) * 8 + 16 +
         kTcStages * sizeof(GemvUnit);
}

int gemv_launch_count(const GemvPlan& p, char trans, int nrhs, int elem_bytes) {
  const GemvSide& side = p.side[(trans == 'N' || trans == 'n') ? 0 : 1];
  int per_tile = 1;  // gather
  for (int c = 0; c < side.nz; ++c) per_tile += side.z[c].ntasks > 0;
  per_tile += side.nzred > 0 && !side.zfused;
  per_tile += side.y.ntasks > 0;
  per_tile += side.nyrows > 0;  // final pass
  const int maxR = elem_bytes >= 16 ? 4 : 16;
  return per_tile * ((nrhs + maxR - 1) / maxR);
}

template <typename T>
void launch_leaf_gradients(const GemvPlan& p, int nrhs, const T* x, const T* r, T* xz, T* rz, T* gfull, T* grk,
                           bool accumulate, GemvStatus* err, cudaStream_t s) {
  constexpr bool big = sizeof(T) < 16;
  if (big && nrhs > 8) grads_tile<T, big ? 16 : 4>(p, nrhs, x, r, xz, rz, gfull, grk, accumulate, err, s);
  else if (big && nrhs > 4) grads_tile<T, big ? 8 : 4>(p, nrhs, x, r, xz, rz, gfull, grk, accumulate, err, s);
  else if (nrhs > 1) grads_tile<T, 4>(p, nrhs, x, r, xz, rz, gfull, grk, accumulate, err, s);
  else grads_tile<T, 1>(p, nrhs, x, r, xz, rz, gfull, grk, accumulate, err, s);
}

template <typename T>
void launch_gemv_adjoint(const GemvPlan& p, int nrhs, const T* x, const T* r, T* dx, T* xz, T* rz, T* gfull, T* grk,
                         bool accumulate, GemvStatus* err, cudaStream_t s) {
  constexpr bool big = sizeof(T) < 16;
  if (big && nrhs > 8) adjoint_tile<T, big ? 16 : 4>(p, nrhs, x, r, dx, xz, rz, gfull, grk, accumulate, err, s);
  else if (big && nrhs > 4) adjoint_tile<T, big ? 8 : 4>(p, nrhs, x, r, dx, xz, rz, gfull, grk, accumulate, err, s);
  else if (nrhs > 1) adjoint_tile<T, 4>(p, nrhs, x, r, dx, xz, rz, gfull, grk, accumulate, err, s);
  else adjoint_tile<T, 1>(p, nrhs, x, r, dx, xz, rz, gfull, grk, accumulate, err, s);
}

template <typename T>
void launch_gemv(const GemvPlan& p, char trans, int nrhs, T alpha, T beta, const T* x_client, T* y_client, T* xz,
                 GemvStatus* err, cudaStream_t s, const GemvTiming* tm) {
  if (trans == 'N') run_all<T, false>(p, nrhs, alpha, beta, x_client, y_client, xz, 0, err, s, tm);
  else
    run_all<T, true>(p, nrhs, alpha, beta, x_client, y_client, xz, (trans == 'C' && Traits<T>::is_complex) ? 1 : 0,
                     err, s, tm);
}

#define HB_INST(T)                                                                                            \
  template void launch_gemv<T>(const GemvPlan&, char, int, T, T, const T*, T*, T*, GemvStatus*, cudaStream_t,         \
                               const GemvTiming*);                                                             \
  template void launch_leaf_gradients<T>(const GemvPlan&, int, const T*, const T*, T*, T*, T*, T*, bool, GemvStatus*, \
                                         cudaStream_t);                                                                  \
  template void launch_gemv_adjoint<T>(const GemvPlan&, int, const T*, const T*, T*, T*, T*, T*, T*, bool, GemvStatus*, \
                                       cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
