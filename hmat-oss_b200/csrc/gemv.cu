// Batched H-matrix-vector product over all leaves, as three launches on device-resident
// schedules (captured together in a CUDA graph by the engine):
//
//   gather   x_rm[i][q] = x[perm[i] + q N]            client -> cluster order, row-major
//   z-phase  z_L = B_L^T x_J (or A_L^T x_I for 'T')     per Rk leaf, long leaves in chunks
//   y-phase  y_I = beta y_I + alpha (sum_F F x_J + sum_Rk A_L[I] z_L)
//                                                       one CTA per row-cluster leaf, so every
//                                                       row of y has exactly one writer; the
//                                                       result is scattered to client order.
//
// This restates HMatrix<T>::gemv (h_matrix.cpp:792-857) with its leaf products
// (ScalarArray::gemm, scalar_array.cpp:413-443; RkMatrix::gemv, rk_matrix.cpp:156-206) and
// the reorderVector / restoreVectorOrder permutations of the C wrapper
// (h_matrix.cpp:75-141, c_wrapping.hpp:233-252).  Summation over the leaves of a row block
// is deterministic (fixed group order), so repeated products are bitwise identical.
#include "gemv_plan.h"
#include "kernels.h"

namespace hmatb200 {
namespace {

constexpr int kZThreads = 128;
constexpr int kYThreads = 128;

template <typename T, int Q>
struct Vec {
  T v[Q];
};

// Loads Q consecutive elements (Q * sizeof(T) bytes, aligned to that size or 16 B).
template <typename T, int Q>
__device__ inline void load_vec(const T* p, T (&out)[Q]) {
  constexpr int bytes = Q * (int)sizeof(T);
  if constexpr (bytes % 16 == 0) {
    const uint4* s = reinterpret_cast<const uint4*>(p);
    uint4* d = reinterpret_cast<uint4*>(out);
#pragma unroll
    for (int c = 0; c < bytes / 16; ++c) d[c] = __ldg(s + c);
  } else if constexpr (bytes % 8 == 0) {
    const uint2* s = reinterpret_cast<const uint2*>(p);
    uint2* d = reinterpret_cast<uint2*>(out);
#pragma unroll
    for (int c = 0; c < bytes / 8; ++c) d[c] = __ldg(s + c);
  } else {
#pragma unroll
    for (int c = 0; c < Q; ++c) out[c] = p[c];
  }
}

template <typename T, bool CONJ>
__device__ inline T maybe_conj(T a) {
  if constexpr (CONJ) return conjg(a);
  else return a;
}

__device__ inline float shfl_xor(float v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ inline double shfl_xor(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ inline cfloat shfl_xor(cfloat v, int m) {
  return cfloat{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}
__device__ inline cdouble shfl_xor(cdouble v, int m) {
  return cdouble{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}

// ---------------------------------------------------------------------------------
template <typename T, int R>
__global__ void gather_kernel(const T* __restrict__ x, int N, int ldx, int q0, int r, const int* __restrict__ perm,
                              T* __restrict__ x_rm) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)N * R) return;
  const int i = (int)(e / R), q = (int)(e % R);
  x_rm[e] = (q0 + q < r) ? x[(size_t)perm[i] + (size_t)(q0 + q) * ldx] : zero<T>();
}

// ---------------------------------------------------------------------------------
// z-phase.  Warp w takes rank columns l = w, w + 4, ...; lanes are RG row groups x QG
// right-hand-side groups of Q values each; partial sums meet through xor shuffles.
template <typename T, int R, bool TRANS, bool CONJ>
__global__ void __launch_bounds__(kZThreads) zphase_kernel(const GemvRkLeaf* __restrict__ rk,
                                                           const GemvZItem* __restrict__ items,
                                                           const T* __restrict__ arena,
                                                           const T* __restrict__ x_rm, T* __restrict__ zout) {
  constexpr int Q = R >= 4 ? 4 : R;
  constexpr int QG = R / Q;
  constexpr int RG = 32 / QG;
  const GemvZItem it = items[blockIdx.x];
  const GemvRkLeaf L = rk[it.leaf];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kZThreads / 32;
  const int rg = lane / QG, qg = lane % QG;
  const T* P;
  int ld, base;
  if constexpr (!TRANS) {
    P = arena + L.off + (size_t)L.m * L.k;  // B, n x k
    ld = L.n;
    base = L.col_off;
  } else {
    P = arena + L.off;  // A, m x k
    ld = L.m;
    base = L.row_off;
  }
  T* dst = zout + it.dst_off;
  for (int l = warp; l < L.k; l += nw) {
    T acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) acc[q] = zero<T>();
    const T* col = P + (size_t)l * ld;
    for (int j = it.start + rg; j < it.start + it.len; j += RG) {
      const T p = maybe_conj<T, CONJ>(col[j]);
      T xv[Q];
      load_vec<T, Q>(x_rm + (size_t)(base + j) * R + qg * Q, xv);
#pragma unroll
      for (int q = 0; q < Q; ++q) acc[q] = fmadd(p, xv[q], acc[q]);
    }
#pragma unroll
    for (int msk = QG; msk < 32; msk <<= 1)
#pragma unroll
      for (int q = 0; q < Q; ++q) acc[q] = acc[q] + shfl_xor(acc[q], msk);
    if (rg == 0) {
#pragma unroll
      for (int q = 0; q < Q; ++q) dst[(size_t)l * R + qg * Q + q] = acc[q];
    }
  }
}

// Sums the chunk partials of long leaves in item order.
template <typename T, int R>
__global__ void zred_kernel(const GemvRkLeaf* __restrict__ rk, const int* __restrict__ multi,
                            const int* __restrict__ mfirst, const int* __restrict__ mcount,
                            const GemvZItem* __restrict__ items, T* __restrict__ z) {
  const int leaf = multi[blockIdx.x];
  const GemvRkLeaf L = rk[leaf];
  const int cnt = mcount[blockIdx.x], first = mfirst[blockIdx.x];
  for (int e = threadIdx.x; e < L.k * R; e += blockDim.x) {
    T s = zero<T>();
    for (int c = 0; c < cnt; ++c) s = s + z[items[first + c].dst_off + e];
    z[L.zoff + e] = s;
  }
}

// ---------------------------------------------------------------------------------
// y-phase.  The CTA owns rows [blk.off, blk.off + blk.len) of the output; its threads form
// NG = blockDim / GS groups of GS threads (one output row per thread) that take the
// block's entries round-robin.  Group partials are summed in group order at the end.
template <typename T, int R, bool TRANS, bool CONJ>
__global__ void __launch_bounds__(kYThreads) yphase_kernel(
    const GemvYBlock* __restrict__ blocks, const GemvYEntry* __restrict__ entries,
    const GemvFullLeaf* __restrict__ full, const GemvRkLeaf* __restrict__ rk, const T* __restrict__ full_arena,
    const T* __restrict__ rk_arena, const T* __restrict__ x_rm, const T* __restrict__ z, int GS,
    const int* __restrict__ perm_out, T* __restrict__ y, int ldy, int q0, int r, T alpha, T beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);
  const GemvYBlock blk = blocks[blockIdx.x];
  const int NG = kYThreads / GS;
  const int g = threadIdx.x / GS;
  for (int r0 = 0; r0 < blk.len; r0 += GS) {
    const int i = r0 + (threadIdx.x % GS);
    const bool active = g < NG && i < blk.len;
    T acc[R];
#pragma unroll
    for (int q = 0; q < R; ++q) acc[q] = zero<T>();
    if (active) {
      for (int e = blk.first + g; e < blk.first + blk.count; e += NG) {
        const GemvYEntry en = entries[e];
        if (en.type == 0) {
          const GemvFullLeaf F = full[en.leaf];
          const T* Fp = full_arena + F.off;
          if constexpr (!TRANS) {
            // rows of F are the block rows: y_i += sum_j F[i, j] x_j
            const T* col = Fp + en.sub + i;
            const T* xr = x_rm + (size_t)F.col_off * R;
            for (int j = 0; j < F.n; ++j) {
              const T f = col[(size_t)j * F.m];
              T xv[R];
              load_vec<T, R>(xr + (size_t)j * R, xv);
#pragma unroll
              for (int q = 0; q < R; ++q) acc[q] = fmadd(f, xv[q], acc[q]);
            }
          } else {
            // columns of F are the block rows: y_j += sum_i op(F[i, j]) x_i
            const T* col = Fp + (size_t)(en.sub + i) * F.m;
            const T* xr = x_rm + (size_t)F.row_off * R;
            for (int ii = 0; ii < F.m; ++ii) {
              const T f = maybe_conj<T, CONJ>(col[ii]);
              T xv[R];
              load_vec<T, R>(xr + (size_t)ii * R, xv);
#pragma unroll
              for (int q = 0; q < R; ++q) acc[q] = fmadd(f, xv[q], acc[q]);
            }
          }
        } else {
          const GemvRkLeaf L = rk[en.leaf];
          const T* P;
          int ld;
          if constexpr (!TRANS) {
            P = rk_arena + L.off;  // A
            ld = L.m;
          } else {
            P = rk_arena + L.off + (size_t)L.m * L.k;  // B
            ld = L.n;
          }
          const T* zl = z + L.zoff;
          const T* row = P + en.sub + i;
          for (int l = 0; l < L.k; ++l) {
            const T p = maybe_conj<T, CONJ>(row[(size_t)l * ld]);
            T zv[R];
            load_vec<T, R>(zl + (size_t)l * R, zv);
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q] = fmadd(p, zv[q], acc[q]);
          }
        }
      }
    }
    // cross-group sum (group order), then scale and scatter to client order
    if (NG > 1) {
      __syncthreads();
      if (active) {
#pragma unroll
        for (int q = 0; q < R; ++q) red[((size_t)g * GS + (threadIdx.x % GS)) * R + q] = acc[q];
      }
      __syncthreads();
      if (g == 0 && active) {
        for (int gg = 1; gg < NG; ++gg)
#pragma unroll
          for (int q = 0; q < R; ++q) acc[q] = acc[q] + red[((size_t)gg * GS + threadIdx.x) * R + q];
      }
    }
    if (g == 0 && active) {
      const size_t dst = (size_t)perm_out[blk.off + i];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if (q0 + q < r) {
          T* yp = y + dst + (size_t)(q0 + q) * ldy;
          T v = alpha * acc[q];
          if (!is_zero_val(beta)) v = fmadd(beta, *yp, v);
          *yp = v;
        }
      }
    }
  }
}

template <typename T, int R, bool TRANS, bool CONJ>
void run_tile(const GemvPlan& p, const GemvSide& side, int nrhs, int q0, T alpha, T beta, const T* x, T* y, T* x_rm,
              T* zpart, T* z, cudaStream_t s, const GemvTiming* tm) {
  if (tm) cudaEventRecord(tm->ev[0], s);
  const int n_in = TRANS ? p.n_rows : p.n_cols;
  const int* perm_in = TRANS ? p.perm_rows : p.perm_cols;
  const int* perm_out = TRANS ? p.perm_cols : p.perm_rows;
  const int ld_in = n_in, ld_out = TRANS ? p.n_cols : p.n_rows;
  long long tot = (long long)n_in * R;
  gather_kernel<T, R><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(x, n_in, ld_in, q0, nrhs, perm_in, x_rm);
  if (tm) cudaEventRecord(tm->ev[1], s);
  if (side.nzitems > 0) {
    // single-item leaves write z directly; chunked leaves write partials
    // single-item leaves write their z in place; chunks of long leaves write partials
    // further down the same buffer, summed by zred
    zphase_kernel<T, R, TRANS, CONJ><<<side.nzitems, kZThreads, 0, s>>>(p.rk, side.zitems,
                                                                        (const T*)p.rk_arena, x_rm, z);
    if (side.nmulti > 0)
      zred_kernel<T, R><<<side.nmulti, 128, 0, s>>>(p.rk, side.multi, side.mfirst, side.mcount, side.zitems, z);
  }
  if (tm) cudaEventRecord(tm->ev[2], s);
  if (side.nblocks > 0) {
    size_t smem = (size_t)kYThreads * R * sizeof(T);
    yphase_kernel<T, R, TRANS, CONJ><<<side.nblocks, kYThreads, smem, s>>>(
        side.blocks, side.entries, p.full, p.rk, (const T*)p.full_arena, (const T*)p.rk_arena, x_rm, z, side.GS,
        perm_out, y, ld_out, q0, nrhs, alpha, beta);
  }
  if (tm) cudaEventRecord(tm->ev[3], s);
}

template <typename T, bool TRANS, bool CONJ>
void run_all(const GemvPlan& p, int nrhs, T alpha, T beta, const T* x, T* y, T* x_rm, T* zpart, T* z,
             cudaStream_t s, const GemvTiming* tm) {
  const GemvSide& side = TRANS ? p.side_t : p.side_n;
  for (int q0 = 0; q0 < nrhs; q0 += 16) {
    const int rem = nrhs - q0;
    if (rem > 8) run_tile<T, 16, TRANS, CONJ>(p, side, nrhs, q0, alpha, beta, x, y, x_rm, zpart, z, s, tm);
    else if (rem > 4) run_tile<T, 8, TRANS, CONJ>(p, side, nrhs, q0, alpha, beta, x, y, x_rm, zpart, z, s, tm);
    else if (rem > 2) run_tile<T, 4, TRANS, CONJ>(p, side, nrhs, q0, alpha, beta, x, y, x_rm, zpart, z, s, tm);
    else if (rem == 2) run_tile<T, 2, TRANS, CONJ>(p, side, nrhs, q0, alpha, beta, x, y, x_rm, zpart, z, s, tm);
    else run_tile<T, 1, TRANS, CONJ>(p, side, nrhs, q0, alpha, beta, x, y, x_rm, zpart, z, s, tm);
  }
}

// ---------------------------------------------------------------------------------
// Leaf-factor gradients (adjoint of y = H x with respect to the stored leaves).
template <typename T, int R>
__global__ void grad_full_kernel(const GemvFullLeaf* __restrict__ full, int nfull, const T* __restrict__ x_rm,
                                 const T* __restrict__ r_rm, T* __restrict__ g, bool accumulate) {
  for (int f = blockIdx.x; f < nfull; f += gridDim.x) {
    const GemvFullLeaf F = full[f];
    T* dF = g + F.off;
    for (int e = threadIdx.x; e < F.m * F.n; e += blockDim.x) {
      const int i = e % F.m, j = e / F.m;
      T rv[R], xv[R];
      load_vec<T, R>(r_rm + (size_t)(F.row_off + i) * R, rv);
      load_vec<T, R>(x_rm + (size_t)(F.col_off + j) * R, xv);
      T acc = accumulate ? dF[e] : zero<T>();
#pragma unroll
      for (int q = 0; q < R; ++q) acc = fmadd(rv[q], xv[q], acc);
      dF[e] = acc;
    }
  }
}

template <typename T, int R>
__global__ void grad_rk_kernel(const GemvRkLeaf* __restrict__ rk, int nrk, const T* __restrict__ x_rm,
                               const T* __restrict__ r_rm, const T* __restrict__ zx, const T* __restrict__ zr,
                               T* __restrict__ g, bool accumulate) {
  for (int t = blockIdx.x; t < nrk; t += gridDim.x) {
    const GemvRkLeaf L = rk[t];
    T* dA = g + L.off;
    T* dB = dA + (size_t)L.m * L.k;
    // dA[i, l] = sum_q r[i, q] z[l, q],  z = B^T x
    for (int e = threadIdx.x; e < L.m * L.k; e += blockDim.x) {
      const int i = e % L.m, l = e / L.m;
      T rv[R], zv[R];
      load_vec<T, R>(r_rm + (size_t)(L.row_off + i) * R, rv);
      load_vec<T, R>(zx + L.zoff + (size_t)l * R, zv);
      T acc = accumulate ? dA[e] : zero<T>();
#pragma unroll
      for (int q = 0; q < R; ++q) acc = fmadd(rv[q], zv[q], acc);
      dA[e] = acc;
    }
    // dB[j, l] = sum_q x[j, q] w[l, q],  w = A^T r
    for (int e = threadIdx.x; e < L.n * L.k; e += blockDim.x) {
      const int j = e % L.n, l = e / L.n;
      T xv[R], wv[R];
      load_vec<T, R>(x_rm + (size_t)(L.col_off + j) * R, xv);
      load_vec<T, R>(zr + L.zoff + (size_t)l * R, wv);
      T acc = accumulate ? dB[e] : zero<T>();
#pragma unroll
      for (int q = 0; q < R; ++q) acc = fmadd(xv[q], wv[q], acc);
      dB[e] = acc;
    }
  }
}

template <typename T, int R>
void grads_tile(const GemvPlan& p, int nrhs, const T* x, const T* r, T* x_rm, T* r_rm, T* zx, T* zr, T* gfull,
                T* grk, bool accumulate, cudaStream_t s) {
  long long tot = (long long)p.n_cols * R;
  gather_kernel<T, R><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(x, p.n_cols, p.n_cols, 0, nrhs, p.perm_cols,
                                                                     x_rm);
  tot = (long long)p.n_rows * R;
  gather_kernel<T, R><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(r, p.n_rows, p.n_rows, 0, nrhs, p.perm_rows,
                                                                     r_rm);
  const GemvSide& sn = p.side_n;
  const GemvSide& st = p.side_t;
  if (sn.nzitems > 0) {
    zphase_kernel<T, R, false, false><<<sn.nzitems, kZThreads, 0, s>>>(p.rk, sn.zitems, (const T*)p.rk_arena, x_rm,
                                                                       zx);
    if (sn.nmulti > 0) zred_kernel<T, R><<<sn.nmulti, 128, 0, s>>>(p.rk, sn.multi, sn.mfirst, sn.mcount, sn.zitems, zx);
  }
  if (st.nzitems > 0) {
    zphase_kernel<T, R, true, false><<<st.nzitems, kZThreads, 0, s>>>(p.rk, st.zitems, (const T*)p.rk_arena, r_rm,
                                                                      zr);
    if (st.nmulti > 0) zred_kernel<T, R><<<st.nmulti, 128, 0, s>>>(p.rk, st.multi, st.mfirst, st.mcount, st.zitems, zr);
  }
  const int grid = persistent_grid(4);
  if (p.nfull > 0 && gfull)
    grad_full_kernel<T, R><<<grid, 256, 0, s>>>(p.full, p.nfull, x_rm, r_rm, gfull, accumulate);
  if (p.nrk > 0 && grk) grad_rk_kernel<T, R><<<grid, 256, 0, s>>>(p.rk, p.nrk, x_rm, r_rm, zx, zr, grk, accumulate);
}

}  // namespace

template <typename T>
void launch_leaf_gradients(const GemvPlan& p, int nrhs, const T* x, const T* r, T* x_rm, T* r_rm, T* zx, T* zr,
                           T* gfull, T* grk, bool accumulate, cudaStream_t s) {
  if (nrhs > 8) grads_tile<T, 16>(p, nrhs, x, r, x_rm, r_rm, zx, zr, gfull, grk, accumulate, s);
  else if (nrhs > 4) grads_tile<T, 8>(p, nrhs, x, r, x_rm, r_rm, zx, zr, gfull, grk, accumulate, s);
  else if (nrhs > 2) grads_tile<T, 4>(p, nrhs, x, r, x_rm, r_rm, zx, zr, gfull, grk, accumulate, s);
  else if (nrhs == 2) grads_tile<T, 2>(p, nrhs, x, r, x_rm, r_rm, zx, zr, gfull, grk, accumulate, s);
  else grads_tile<T, 1>(p, nrhs, x, r, x_rm, r_rm, zx, zr, gfull, grk, accumulate, s);
}

template <typename T>
void launch_gemv(const GemvPlan& p, char trans, int nrhs, T alpha, T beta, const T* x_client, T* y_client,
                 T* x_rm, T* zpart, T* z, cudaStream_t s, const GemvTiming* tm) {
  if (trans == 'N') run_all<T, false, false>(p, nrhs, alpha, beta, x_client, y_client, x_rm, zpart, z, s, tm);
  else if (trans == 'T' || !Traits<T>::is_complex)
    run_all<T, true, false>(p, nrhs, alpha, beta, x_client, y_client, x_rm, zpart, z, s, tm);
  else run_all<T, true, true>(p, nrhs, alpha, beta, x_client, y_client, x_rm, zpart, z, s, tm);
}

#define HB_INST(T)                                                                                          \
  template void launch_gemv<T>(const GemvPlan&, char, int, T, T, const T*, T*, T*, T*, T*, cudaStream_t,         \
                               const GemvTiming*);                                                             \
  template void launch_leaf_gradients<T>(const GemvPlan&, int, const T*, const T*, T*, T*, T*, T*, T*, T*, bool, \
                                         cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
