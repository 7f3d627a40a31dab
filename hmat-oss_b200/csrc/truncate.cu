// Batched Rk truncation in FP64, one CTA per leaf on a persistent grid.
//
// Restates RkMatrix<T>::truncate (rk_matrix.cpp:490-585) for k <= min(m, n):
//   A = Qa Ra, B = Qb Rb                         (qrDecomposition, scalar_array.cpp:1083-1133)
//   Ra Rb^T = U S V^H                            (truncatedSvdDecomposition, scalar_array.cpp:927-966)
//   k' = #{ sigma_i > eps sigma_0 }               (findK, scalar_array.cpp:97-115)
//   A' = Qa [U_k' sqrt(S); 0],  B' = Qb [conj(V_k') sqrt(S); 0]   (truncatedAB, rk_matrix.cpp:265-297)
// QR is Householder (column norms and panel updates as warp reductions), the SVD of the
// small core is one-sided Jacobi with a round-robin pair schedule; both run in FP64 (or
// complex FP64) whatever the storage type, and the new factors are narrowed back into the
// leaf's workspace slot.
#include <cstdlib>

#include "block_reduce.cuh"
#include "kernels.h"

namespace hmatb200 {
namespace {

constexpr int kTruncThreads = 256;
// Cap on the one-sided Jacobi sweeps of a core SVD (a leaf that reaches it is flagged
// kLeafSvdNoConverge and its assembly fails).  Set by the host before each assembly.
__device__ int g_jacobi_max_sweeps = kJacobiDefaultSweeps;

__device__ inline double sqrt_abs2(double a) { return fabs(a); }
__device__ inline double sqrt_abs2(cdouble a) { return sqrt(a.x * a.x + a.y * a.y); }
__device__ inline double phase_of(double a, double absa) { return absa == 0.0 ? 1.0 : a / absa; }
__device__ inline cdouble phase_of(cdouble a, double absa) {
  return absa == 0.0 ? cdouble{1.0, 0.0} : cdouble{a.x / absa, a.y / absa};
}
__device__ inline double scal(double s, double a) { return s * a; }
__device__ inline cdouble scal(double s, cdouble a) { return cdouble{s * a.x, s * a.y}; }

// Householder QR of X (len x k, ld = len) in place: v_j stored in X[j:, j] (v_j[j] explicit),
// tau[j], and R (k x k, column-major, upper) written separately.
template <typename W>
__device__ void householder_qr(W* X, int len, int k, W* tau, W* R, RedScratch& rs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = 0; j < k; ++j) {
    W* x = X + (size_t)j * len;
    double nrm2 = 0.0;
    for (int i = j + threadIdx.x; i < len; i += blockDim.x) nrm2 += abs2(x[i]);
    nrm2 = block_sum(nrm2, rs);
    const double nrm = sqrt(nrm2);
    const W alpha = x[j];
    const double aa = sqrt_abs2(alpha);
    W beta = scal(-nrm, phase_of(alpha, aa));
    W t = zero<W>();
    if (nrm > 0.0) {
      W v0 = alpha - beta;
      double vn2 = nrm2 - aa * aa + abs2(v0);
      t = vn2 > 0.0 ? scal(2.0 / vn2, one<W>()) : zero<W>();
      __syncthreads();
      if (threadIdx.x == 0) x[j] = v0;
      __syncthreads();
    } else {
      beta = zero<W>();
    }
    if (threadIdx.x == 0) {
      tau[j] = t;
      R[j + (size_t)j * k] = beta;
      for (int i = j + 1; i < k; ++i) R[i + (size_t)j * k] = zero<W>();
    }
    // apply H_j = I - t v v^H to columns c > j, warp per column
    for (int c = j + 1 + warp; c < k; c += nw) {
      W* y = X + (size_t)c * len;
      W s = zero<W>();
      if (nrm > 0.0)
        for (int i = j + lane; i < len; i += 32) s = s + conjg(x[i]) * y[i];
      s = warp_sum(s);
      s = warp_bcast(s);
      W ts = t * s;
      if (nrm > 0.0)
        for (int i = j + lane; i < len; i += 32) y[i] = y[i] - ts * x[i];
      __syncwarp();
      if (lane == 0) R[j + (size_t)c * k] = y[j];
    }
    __syncthreads();
  }
}

// C[:, c] <- H_0 ... H_{k-1} C[:, c] for every column, warp per column (Q applied to the
// k x k' block stacked on zeros).
template <typename W>
__device__ void apply_q(const W* X, int len, int k, const W* tau, W* C, int ncols) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = warp; c < ncols; c += nw) {
    W* y = C + (size_t)c * len;
    for (int h = k - 1; h >= 0; --h) {
      const W* v = X + (size_t)h * len;
      W s = zero<W>();
      for (int i = h + lane; i < len; i += 32) s = s + conjg(v[i]) * y[i];
      s = warp_sum(s);
      s = warp_bcast(s);
      W ts = tau[h] * s;
      for (int i = h + lane; i < len; i += 32) y[i] = y[i] - ts * v[i];
      __syncwarp();
    }
  }
  __syncthreads();
}

// One-sided Jacobi on the k x k matrix Wm (in place), accumulating V.  On return the
// columns of Wm are U_j sigma_j (unsorted).  Returns false if the sweep cap was hit.
template <typename W>
__device__ bool jacobi_svd(W* Wm, W* V, int k, RedScratch& rs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = threadIdx.x; i < k * k; i += blockDim.x) V[i] = (i % (k + 1) == 0) ? one<W>() : zero<W>();
  __syncthreads();
  const int kk = (k + 1) & ~1;  // even number of players (the extra one sits out)
  const int max_sweeps = g_jacobi_max_sweeps;
  __shared__ int s_rot;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) s_rot = 0;
    __syncthreads();
    for (int round = 0; round < kk - 1; ++round) {
      for (int pr = warp; pr < kk / 2; pr += nw) {
        // circle method: player 0 fixed, the others rotate
        int a = pr == 0 ? 0 : 1 + (pr - 1 + round) % (kk - 1);
        int b = 1 + (kk - 2 - pr + round) % (kk - 1);
        int p = min(a, b), q = max(a, b);
        if (q >= k) continue;
        W* wp = Wm + (size_t)p * k;
        W* wq = Wm + (size_t)q * k;
        double al = 0.0, be = 0.0;
        W g = zero<W>();
        for (int i = lane; i < k; i += 32) {
          al += abs2(wp[i]);
          be += abs2(wq[i]);
          g = g + conjg(wp[i]) * wq[i];
        }
        al = warp_sum(al);
        be = warp_sum(be);
        g = warp_sum(g);
        al = __shfl_sync(0xffffffffu, al, 0);
        be = __shfl_sync(0xffffffffu, be, 0);
        g = warp_bcast(g);
        double ag = sqrt(abs2(g));
        if (ag == 0.0 || ag <= 1e-15 * sqrt(al * be)) continue;
        if (lane == 0) s_rot = 1;
        W ph = scal(1.0 / ag, g);  // e^{i phi}
        double zeta = (be - al) / (2.0 * ag);
        double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        W phc = conjg(ph);
        W* vp = V + (size_t)p * k;
        W* vq = V + (size_t)q * k;
        for (int i = lane; i < k; i += 32) {
          W x = wp[i], y = wq[i] * phc;
          wp[i] = scal(cs, x) - scal(sn, y);
          wq[i] = scal(sn, x) + scal(cs, y);
          W vx = vp[i], vy = vq[i] * phc;
          vp[i] = scal(cs, vx) - scal(sn, vy);
          vq[i] = scal(sn, vx) + scal(cs, vy);
        }
      }
      __syncthreads();
    }
    if (!s_rot) return true;
    __syncthreads();
  }
  return false;
}

template <typename T>
__global__ void __launch_bounds__(kTruncThreads) truncate_kernel(const RkLeafDesc* __restrict__ leaves,
                                                                 const int* __restrict__ order, int nleaves,
                                                                 double eps, T* ws, int* ranks, int* status,
                                                                 int* counter, typename Traits<T>::wide* scratch,
                                                                 long long slab_elems) {
  typedef typename Traits<T>::wide W;
  __shared__ RedScratch rs;
  __shared__ int s_item;
  __shared__ int s_newk;
  W* slab = scratch + (size_t)blockIdx.x * slab_elems;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nleaves) break;
    const int leaf = order[item];
    const RkLeafDesc d = leaves[leaf];
    const int m = d.m, n = d.n, k = ranks[leaf];
    if (k <= 0) continue;
    T* A = ws + d.ws_off;
    T* B = A + (size_t)m * d.kcap;
    // slab layout
    W* Wa = slab;
    W* Wb = Wa + (size_t)m * k;
    W* Ca = Wb + (size_t)n * k;
    W* Cb = Ca + (size_t)m * k;
    W* Ra = Cb + (size_t)n * k;
    W* Rb = Ra + (size_t)k * k;
    W* Rm = Rb + (size_t)k * k;
    W* Vm = Rm + (size_t)k * k;
    W* tau_a = Vm + (size_t)k * k;
    W* tau_b = tau_a + k;
    double* sig = reinterpret_cast<double*>(tau_b + k);
    int* ord = reinterpret_cast<int*>(sig + k);

    for (size_t e = threadIdx.x; e < (size_t)m * k; e += blockDim.x) Wa[e] = widen(A[e]);
    for (size_t e = threadIdx.x; e < (size_t)n * k; e += blockDim.x) Wb[e] = widen(B[e]);
    __syncthreads();
    householder_qr(Wa, m, k, tau_a, Ra, rs);
    householder_qr(Wb, n, k, tau_b, Rb, rs);
    // Rm = Ra Rb^T (both upper triangular)
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
      int i = e % k, j = e / k;
      W s = zero<W>();
      for (int l = max(i, j); l < k; ++l) s = s + Ra[i + (size_t)l * k] * Rb[j + (size_t)l * k];
      Rm[e] = s;
    }
    __syncthreads();
    bool conv = jacobi_svd(Rm, Vm, k, rs);
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      double s2 = 0.0;
      for (int i = 0; i < k; ++i) s2 += abs2(Rm[i + (size_t)j * k]);
      sig[j] = sqrt(s2);
    }
    __syncthreads();
    // descending order, ties by index (stable)
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      int r = 0;
      for (int i = 0; i < k; ++i) r += (sig[i] > sig[j]) || (sig[i] == sig[j] && i < j);
      ord[r] = j;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double thr = sig[ord[0]] * eps;
      int nk = 0;
      while (nk < k && !(sig[ord[nk]] <= thr)) nk++;
      s_newk = nk;
    }
    __syncthreads();
    const int nk = s_newk;
    // Ca = [U_k' sqrt(S); 0], Cb = [conj(V_k') sqrt(S); 0]
    for (size_t e = threadIdx.x; e < (size_t)m * nk; e += blockDim.x) {
      int i = (int)(e % m), c = (int)(e / m);
      int o = ord[c];
      double sc = sig[o];
      Ca[e] = (i < k && sc > 0.0) ? scal(1.0 / sqrt(sc), Rm[i + (size_t)o * k]) : zero<W>();
    }
    for (size_t e = threadIdx.x; e < (size_t)n * nk; e += blockDim.x) {
      int i = (int)(e % n), c = (int)(e / n);
      int o = ord[c];
      Cb[e] = i < k ? scal(sqrt(sig[o]), conjg(Vm[i + (size_t)o * k])) : zero<W>();
    }
    __syncthreads();
    apply_q(Wa, m, k, tau_a, Ca, nk);
    apply_q(Wb, n, k, tau_b, Cb, nk);
    for (size_t e = threadIdx.x; e < (size_t)m * nk; e += blockDim.x) A[e] = narrow<T>(Ca[e]);
    for (size_t e = threadIdx.x; e < (size_t)n * nk; e += blockDim.x) B[e] = narrow<T>(Cb[e]);
    __syncthreads();
    if (threadIdx.x == 0) {
      ranks[leaf] = nk;
      if (!conv && status[leaf] == kLeafOk) status[leaf] = kLeafSvdNoConverge;
    }
  }
}

// Writes A as row panels (len x k column-major each) and B transposed (k x n column-major,
// leading dimension bt_ld: rows of a taller matrix of stacked B^T blocks).
template <typename T>
__global__ void compact_kernel(const RkLeafDesc* __restrict__ leaves, int nleaves, const T* __restrict__ ws,
                               const int* __restrict__ ranks, const RkStoreDesc* __restrict__ store,
                               const PanelDesc* __restrict__ panels, T* arena) {
  const int leaf = blockIdx.x;
  if (leaf >= nleaves) return;
  const RkLeafDesc d = leaves[leaf];
  const int k = ranks[leaf];
  if (k <= 0) return;
  const RkStoreDesc st = store[leaf];
  const T* A = ws + d.ws_off;
  const T* B = A + (size_t)d.m * d.kcap;
  for (int p = 0; p < st.npanel; ++p) {
    const PanelDesc P = panels[st.panel_first + p];
    T* dst = arena + P.off;
    for (int e = threadIdx.x; e < P.len * k; e += blockDim.x) {
      const int i = e % P.len, l = e / P.len;
      dst[e] = A[(size_t)l * d.m + P.rs + i];
    }
  }
  T* bt = arena + st.bt_off;
  const int ld = st.bt_ld > 0 ? st.bt_ld : k;
  for (int e = threadIdx.x; e < d.n * k; e += blockDim.x) {
    const int l = e % k, j = e / k;
    bt[l + (size_t)j * ld] = B[(size_t)l * d.n + j];
  }
}

// Inverse of compact_kernel: a leaf's A row panels and B^T back into its workspace slot
// (A m x kcap then B n x kcap, column-major), for re-truncating assembled leaves.
template <typename T>
__global__ void unpack_kernel(const RkLeafDesc* __restrict__ leaves, int nleaves, const int* __restrict__ ranks,
                              const RkStoreDesc* __restrict__ store, const PanelDesc* __restrict__ panels,
                              const T* __restrict__ arena, T* ws) {
  const int leaf = blockIdx.x;
  if (leaf >= nleaves) return;
  const RkLeafDesc d = leaves[leaf];
  const int k = ranks[leaf];
  if (k <= 0) return;
  const RkStoreDesc st = store[leaf];
  T* A = ws + d.ws_off;
  T* B = A + (size_t)d.m * d.kcap;
  for (int p = 0; p < st.npanel; ++p) {
    const PanelDesc P = panels[st.panel_first + p];
    const T* src = arena + P.off;
    for (int e = threadIdx.x; e < P.len * k; e += blockDim.x) {
      const int i = e % P.len, l = e / P.len;
      A[(size_t)l * d.m + P.rs + i] = src[e];
    }
  }
  const T* bt = arena + st.bt_off;
  const int ld = st.bt_ld > 0 ? st.bt_ld : k;
  for (int e = threadIdx.x; e < d.n * k; e += blockDim.x) {
    const int l = e % k, j = e / k;
    B[(size_t)l * d.n + j] = bt[l + (size_t)j * ld];
  }
}

// ---------------------------------------------------------------------------------
// Tall-skinny truncation (every Rk leaf of rank <= 16 real / 8 complex that is not a
// dense-SVD job).
//
// Only the triangular factors of the two QRs are formed.  With A = Qa Ra, B = Qb Rb and the
// core Ra Rb^T = U S V^H (one-sided Jacobi returns W = Ra Rb^T V = U S and V),
//   A' = Qa U_k' S^1/2       = A (Rb^T V_k' S^-1/2)
//   B' = Qb conj(V_k') S^1/2 = B (Ra^T conj(U_k') S^-1/2) = B (Ra^T conj(W_k') S^-3/2)
// since Ra Rb^T V = U S and Rb Ra^T conj(U) = conj(V) S.  The new factors are A and B times
// k x k' maps and no orthogonal factor is ever applied.  The product A' B'^T is the
// reference's truncation (rk_matrix.cpp:490-585) up to rounding of order k u sigma_0, and
// k' comes from the singular values of the same core (findK, scalar_array.cpp:97-115).
//
// The triangles come from a communication-avoiding Householder QR: one warp reduces a row
// segment of a factor (kTsSegRows rows) chunk by chunk, [R; chunk] -> R, the chunk in
// registers (lane l holds rows l, l + 32, ...) and column c of R in lane c; a factor with
// several segments stacks the segment triangles and reduces the stack the same way.  The
// phases (one launch per rank bucket, warp per item):
//   tsqr (segments) -> tsqr (stacks) -> core (Jacobi, findK, maps) -> apply (A M, B M).
constexpr int kTsWarps = 4;

__device__ inline double ts_xor(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ inline cdouble ts_xor(cdouble v, int m) {
  return cdouble{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}

// Per-warp shared memory of the tsqr phase: the next chunk (raw source scalars, column
// major, filled by cp.async while the current chunk is reduced), the partial dot products of
// one Householder step (lane x column), their column sums, and R (row-major, padded).
template <typename W, typename S, int K, int RPL>
struct TsqrSmem {
  S stage[K][32 * RPL];
  W red[32][K + 1];
  W sv[32];
  W R[K][K + 1];
};

__device__ inline void ts_cp_async(void* dst, const void* src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (bytes == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ inline void ts_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ inline void ts_cp_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Issues the copies of rows [r0, r0 + 32 RPL) x columns [0, k) of an item into the stage;
// each lane copies the rows it will read.
template <typename W, typename S, int K, int RPL>
__device__ __forceinline__ void ts_prefetch(TsqrSmem<W, S, K, RPL>& sm, const S* base, int ld, int rows, int k,
                                            int r0, int lane) {
#pragma unroll
  for (int r = 0; r < RPL; ++r) {
    const int row = r0 + r * 32 + lane;
    if (row < rows)
      for (int j = 0; j < k; ++j) ts_cp_async(&sm.stage[j][r * 32 + lane], base + (size_t)j * ld + row, sizeof(S));
  }
  ts_cp_commit();
}

// Householder step J of [R; chunk] -> R, then the steps after it (J is a compile-time
// index so the chunk stays in registers).  The partial dot products of the chunk's column J
// with the columns right of it are summed through shared memory: each lane stores its
// partials, lane l adds up column J + 1 + (l mod 16) over half of the lanes, one exchange
// joins the halves.
template <typename W, typename S, int K, int RPL, int J>
__device__ __forceinline__ void ts_house(W (&c)[RPL][K], TsqrSmem<W, S, K, RPL>& sm, int lane) {
  if constexpr (J < K) {
    constexpr int n = K - 1 - J;
    double p2 = 0.0;
#pragma unroll
    for (int r = 0; r < RPL; ++r) p2 += abs2(c[r][J]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) p2 += __shfl_xor_sync(0xffffffffu, p2, off);
    if (p2 != 0.0) {  // warp-uniform: the butterfly leaves the same sum in every lane
      const W alpha = sm.R[J][J];
      const double aa = sqrt_abs2(alpha);
      const double nrm = sqrt(aa * aa + p2);
      const W beta = scal(-nrm, phase_of(alpha, aa));
      const W v0 = alpha - beta;
      const double t = 2.0 / (p2 + abs2(v0));
      W rnew[n > 0 ? n : 1];
      if constexpr (n > 0) {
#pragma unroll
        for (int col = J + 1; col < K; ++col) {
          W s = zero<W>();
#pragma unroll
          for (int r = 0; r < RPL; ++r) s = s + conjg(c[r][J]) * c[r][col];
          sm.red[lane][col] = s;
        }
        __syncwarp();
        if constexpr (n <= 16) {
          const int q = lane & 15, h = lane >> 4;
          W s = zero<W>();
          if (q < n) {
#pragma unroll
            for (int i = 0; i < 16; ++i) s = s + sm.red[h * 16 + i][J + 1 + q];
          }
          s = s + ts_xor(s, 16);
          if (h == 0 && q < n) sm.sv[q] = s;
        } else {
          W s = zero<W>();
          if (lane < n) {
#pragma unroll 8
            for (int i = 0; i < 32; ++i) s = s + sm.red[i][J + 1 + lane];
            sm.sv[lane] = s;
          }
        }
        __syncwarp();
#pragma unroll
        for (int col = J + 1; col < K; ++col) {
          const W rjc = sm.R[J][col];
          const W ts = scal(t, sm.sv[col - J - 1] + conjg(v0) * rjc);
          rnew[col - J - 1] = rjc - ts * v0;
#pragma unroll
          for (int r = 0; r < RPL; ++r) c[r][col] = c[r][col] - ts * c[r][J];
        }
      }
      __syncwarp();
      if (lane == 0) {
        sm.R[J][J] = beta;
#pragma unroll
        for (int col = J + 1; col < K; ++col) sm.R[J][col] = rnew[col - J - 1];
      }
      __syncwarp();
    }
    ts_house<W, S, K, RPL, J + 1>(c, sm, lane);
  }
}

// R (K x K) of the rows of one item, written column-major with leading dimension ld_r.
// A column whose part below the diagonal is already zero is left as it is (H_j = I, as
// LAPACK's larfg does for real data).
template <typename W, typename S, int K, int RPL, int NW>
__global__ void __launch_bounds__(NW * 32) tsqr_kernel(const TsItem* __restrict__ items, int nitems, const S* src,
                                                        W* tri) {
  extern __shared__ __align__(16) unsigned char ts_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  TsqrSmem<W, S, K, RPL>& sm = reinterpret_cast<TsqrSmem<W, S, K, RPL>*>(ts_smem)[warp];
  constexpr int CH = 32 * RPL;
  const int nwarps = gridDim.x * NW;
  for (int it = blockIdx.x * NW + warp; it < nitems; it += nwarps) {
    const TsItem d = items[it];
    const int k = d.k;
    const S* base = src + d.src;
    __syncwarp();
    for (int e = lane; e < K * (K + 1); e += 32) (&sm.R[0][0])[e] = zero<W>();
    ts_prefetch(sm, base, d.ld, d.rows, k, 0, lane);
    __syncwarp();
    for (int r0 = 0; r0 < d.rows; r0 += CH) {
      ts_cp_wait();  // each lane reads back only the elements it copied
      W c[RPL][K];
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int row = r0 + r * 32 + lane;
#pragma unroll
        for (int j = 0; j < K; ++j) c[r][j] = (row < d.rows && j < k) ? widen(sm.stage[j][r * 32 + lane]) : zero<W>();
      }
      __syncwarp();  // the stage is read before the next copies overwrite it
      if (r0 + CH < d.rows) ts_prefetch(sm, base, d.ld, d.rows, k, r0 + CH, lane);
      ts_house<W, S, K, RPL, 0>(c, sm, lane);
    }
    __syncwarp();
    W* out = tri + d.r_out;
    for (int e = lane; e < K * K; e += 32) {
      const int i = e % K, cc = e / K;
      out[(size_t)cc * d.ld_r + i] = sm.R[i][cc];
    }
  }
}

// Core of a leaf: W = Ra Rb^T V by one-sided Jacobi (the circle schedule of the other
// truncation kernels), k', and the two maps (K x K, rows >= k and columns >= k' zero).  A
// leaf takes K lanes (lane j of the group holds column j of W and of V), so a warp holds
// 32 / K leaves; every shuffle is executed by the whole warp with width K, and a group whose
// leaf has converged (or that has no leaf) computes along without rotating.
__device__ inline double wt_shfl_w(double v, int src, int w) { return __shfl_sync(0xffffffffu, v, src, w); }
__device__ inline cdouble wt_shfl_w(cdouble v, int src, int w) {
  return cdouble{__shfl_sync(0xffffffffu, v.x, src, w), __shfl_sync(0xffffffffu, v.y, src, w)};
}

template <typename W, int K, int NW>
__global__ void __launch_bounds__(NW * 32) tscore_kernel(const TsCore* __restrict__ items, int nitems,
                                                          const W* __restrict__ tri, W* __restrict__ maps,
                                                          int* ranks, int* status, double eps) {
  constexpr int G = 32 / K;  // leaves per warp
  constexpr int SW = (K & (K - 1)) == 0 ? K : 32;  // shuffle width (a power of two; one leaf a warp otherwise)
  __shared__ W s_ra[NW][G][K * K];
  __shared__ W s_rb[NW][G][K * K];
  __shared__ signed char s_partner[NW][K][32];
  __shared__ int s_ord[NW][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane / K, j = lane % K;  // leaf slot in the warp, column in the leaf
  W* Ra = s_ra[warp][grp < G ? grp : 0];
  W* Rb = s_rb[warp][grp < G ? grp : 0];
  int* ord = s_ord[warp] + grp * K;
  const int nwarps = gridDim.x * NW;
  for (int base = (blockIdx.x * NW + warp) * G; base < nitems; base += nwarps * G) {
    const int it = base + grp;
    const bool live = grp < G && it < nitems;
    TsCore d{};
    if (live) d = items[it];
    const int k = live ? d.k : 0;
    __syncwarp();
    if (live)
      for (int e = j; e < K * K; e += K) {
        Ra[e] = tri[d.ra + e];
        Rb[e] = tri[d.rb + e];
      }
    // the circle schedule of this leaf's rank (player 0 fixed, the others rotate)
    const int kk = (k + 1) & ~1;
    if (j < kk)
      for (int round = 0; round < kk - 1; ++round) {
        int partner = -1;
        for (int pr = 0; pr < kk / 2; ++pr) {
          const int a = pr == 0 ? 0 : 1 + (pr - 1 + round) % (kk - 1);
          const int b = 1 + (kk - 2 - pr + round) % (kk - 1);
          if (a == j) partner = b;
          if (b == j) partner = a;
        }
        s_partner[warp][round][lane] = (signed char)partner;
      }
    __syncwarp();
    // column j of Ra Rb^T (rows < k), and of V = I
    W w[K], v[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      W s = zero<W>();
      if (j < k && i < k)
        for (int l = max(i, j); l < k; ++l) s = s + Ra[i + l * K] * Rb[j + l * K];
      w[i] = s;
      v[i] = (i == j) ? one<W>() : zero<W>();
    }
    // rounds of the warp: the largest schedule among its leaves
    int rounds = kk - 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) rounds = max(rounds, __shfl_xor_sync(0xffffffffu, rounds, off));
    bool conv = false;
    const int max_sweeps = g_jacobi_max_sweeps;
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      bool rot = false;
      for (int round = 0; round < rounds; ++round) {
        const int partner = (j < kk && round < kk - 1) ? (int)s_partner[warp][round][lane] : -1;
        const int src = partner < 0 ? j : partner;
        W pw[K];
#pragma unroll
        for (int i = 0; i < K; ++i) pw[i] = wt_shfl_w(w[i], src, SW);
        const bool pair = partner >= 0 && j < k && partner < k;
        const bool is_p = j < partner;
        // both lanes of a pair sum the same squares in the same order; <p, q> is formed on
        // the p lane and sent to the q lane, so both rotate with identical coefficients
        double n_own = 0.0, n_oth = 0.0;
        W g_own = zero<W>();
#pragma unroll
        for (int i = 0; i < K; ++i) {
          n_own += abs2(w[i]);
          n_oth += abs2(pw[i]);
          g_own = g_own + conjg(w[i]) * pw[i];
        }
        const W g_p = wt_shfl_w(g_own, src, SW);
        const double al = is_p ? n_own : n_oth, be = is_p ? n_oth : n_own;
        const W g = is_p ? g_own : g_p;
        const double ag = sqrt(abs2(g));
        const bool do_rot = pair && !conv && !(ag == 0.0 || ag <= 1e-15 * sqrt(al * be));
        rot |= do_rot;
        double cs = 1.0, sn = 0.0;
        W phc = one<W>();
        if (do_rot) {
          const W ph = scal(1.0 / ag, g);
          const double zeta = (be - al) / (2.0 * ag);
          const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          cs = 1.0 / sqrt(1.0 + tt * tt);
          sn = cs * tt;
          phc = conjg(ph);
#pragma unroll
          for (int i = 0; i < K; ++i) {
            const W x = is_p ? w[i] : pw[i];
            const W y = (is_p ? pw[i] : w[i]) * phc;
            w[i] = is_p ? scal(cs, x) - scal(sn, y) : scal(sn, x) + scal(cs, y);
          }
        }
#pragma unroll
        for (int i = 0; i < K; ++i) pw[i] = wt_shfl_w(v[i], src, SW);
        if (do_rot) {
#pragma unroll
          for (int i = 0; i < K; ++i) {
            const W x = is_p ? v[i] : pw[i];
            const W y = (is_p ? pw[i] : v[i]) * phc;
            v[i] = is_p ? scal(cs, x) - scal(sn, y) : scal(sn, x) + scal(cs, y);
          }
        }
      }
      // this leaf has converged when its group made no rotation in a whole sweep
      const unsigned gmask = (K == 32 ? 0xffffffffu : ((1u << K) - 1u)) << (grp * K);
      const unsigned any = __ballot_sync(0xffffffffu, rot);
      if (!(any & gmask)) conv = true;
      if (__all_sync(0xffffffffu, conv)) break;
    }
    // singular values (column norms), descending order with ties by index
    double sg = 0.0;
#pragma unroll
    for (int i = 0; i < K; ++i) sg += abs2(w[i]);
    sg = sqrt(sg);
    int rnk = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const double si = __shfl_sync(0xffffffffu, sg, i, SW);
      if (i < k) rnk += (si > sg) || (si == sg && i < j);
    }
    if (j < k) ord[rnk] = j;
    __syncwarp();
    int nk = 0;
    {
      const double thr = __shfl_sync(0xffffffffu, sg, k > 0 ? ord[0] : j, SW) * eps;
      bool run = true;
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const double si = __shfl_sync(0xffffffffu, sg, i < k ? ord[i] : j, SW);
        run = run && i < k && !(si <= thr);
        nk += run ? 1 : 0;
      }
    }
    // Ma[:, c] = Rb^T V[:, o] / sqrt(s_o), Mb[:, c] = Ra^T conj(W[:, o]) / s_o^3/2 (lane = row)
    for (int c = 0; c < K; ++c) {
      const int o = c < nk ? ord[c] : j;
      const double so = __shfl_sync(0xffffffffu, sg, o, SW);
      W ma = zero<W>(), mb = zero<W>();
#pragma unroll
      for (int l = 0; l < K; ++l) {
        const W vl = wt_shfl_w(v[l], o, SW), wl = wt_shfl_w(w[l], o, SW);
        if (c < nk && j < k && l <= j) {
          ma = ma + Rb[l + j * K] * vl;
          mb = mb + Ra[l + j * K] * conjg(wl);
        }
      }
      if (c < nk) {
        const double rs = 1.0 / sqrt(so);
        ma = scal(rs, ma);
        mb = scal(rs / so, mb);
      }
      if (live) {
        maps[d.ma + (size_t)c * K + j] = ma;
        maps[d.mb + (size_t)c * K + j] = mb;
      }
    }
    if (live && j == 0) {
      ranks[d.leaf] = nk;
      if (!conv && status[d.leaf] == kLeafOk) status[d.leaf] = kLeafSvdNoConverge;
    }
  }
}

// New factor columns in place: rows of the segment times the K x K map, the first k'
// columns written back narrowed.
template <typename T, typename W, int K, int RPL>
__global__ void __launch_bounds__(kTsWarps * 32) tsapply_kernel(const TsItem* __restrict__ items, int nitems,
                                                                 T* ws, const W* __restrict__ maps,
                                                                 const int* __restrict__ ranks) {
  __shared__ W s_map[kTsWarps][K * K];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  W* M = s_map[warp];
  const int nwarps = gridDim.x * kTsWarps;
  for (int it = blockIdx.x * kTsWarps + warp; it < nitems; it += nwarps) {
    const TsItem d = items[it];
    const int k = d.k, nk = ranks[d.leaf];
    if (nk <= 0) continue;
    __syncwarp();
    for (int e = lane; e < K * K; e += 32) M[e] = maps[d.map + e];
    __syncwarp();
    T* base = ws + d.src;
    for (int r0 = 0; r0 < d.rows; r0 += 32 * RPL) {
      W a[RPL][K];
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int row = r0 + r * 32 + lane;
#pragma unroll
        for (int l = 0; l < K; ++l)
          a[r][l] = (row < d.rows && l < k) ? widen(base[(size_t)l * d.ld + row]) : zero<W>();
      }
#pragma unroll
      for (int c = 0; c < K; ++c) {
        if (c >= nk) break;
        W o[RPL];
#pragma unroll
        for (int r = 0; r < RPL; ++r) o[r] = zero<W>();
#pragma unroll
        for (int l = 0; l < K; ++l) {
          const W mlc = M[l + c * K];
#pragma unroll
          for (int r = 0; r < RPL; ++r) o[r] = o[r] + a[r][l] * mlc;
        }
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
          const int row = r0 + r * 32 + lane;
          if (row < d.rows) base[(size_t)c * d.ld + row] = narrow<T>(o[r]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------------
// Tall-skinny truncation of the leaves above the register buckets (rank > 32 real / 16
// complex, not dense-SVD jobs): the same algorithm as tsqr / tscore / tsapply (triangles of
// row segments, stacks of triangles, core, factors times maps), each item taken by a CTA of
// kTruncThreads threads with the CTA-level Householder QR and one-sided Jacobi of
// truncate_kernel on an FP64 slab of its own.  Segments hold at least k rows.

// Triangle of one item: rows x k (ld d.ld) widened into the slab, Householder QR, R written
// with leading dimension d.ld_r.
template <typename W, typename S>
__global__ void __launch_bounds__(kTruncThreads) tsqr_cta_kernel(const TsItem* __restrict__ items, int nitems,
                                                                  const S* src, W* tri, W* scratch,
                                                                  long long slab_elems, int* counter) {
  __shared__ RedScratch rs;
  __shared__ int s_item;
  W* slab = scratch + (size_t)blockIdx.x * slab_elems;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    const TsItem d = items[item];
    const int k = d.k, rows = d.rows;
    W* X = slab;
    W* tau = X + (size_t)rows * k;
    W* R = tau + k;
    for (size_t e = threadIdx.x; e < (size_t)rows * k; e += blockDim.x) {
      const int c = (int)(e / rows), i = (int)(e % rows);
      X[e] = widen(src[d.src + (size_t)c * d.ld + i]);
    }
    __syncthreads();
    householder_qr(X, rows, k, tau, R, rs);
    __syncthreads();
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
      const int i = e % k, c = e / k;
      tri[d.r_out + (size_t)c * d.ld_r + i] = R[e];
    }
  }
}

// Core of one leaf: Ra Rb^T, Jacobi, sigma order, k', and the maps (k x k, ld k, columns at
// or past k' zero), as tscore_kernel.
template <typename W>
__global__ void __launch_bounds__(kTruncThreads) tscore_cta_kernel(const TsCore* __restrict__ items, int nitems,
                                                                    const W* __restrict__ tri, W* maps, int* ranks,
                                                                    int* status, double eps, W* scratch,
                                                                    long long slab_elems, int* counter) {
  __shared__ RedScratch rs;
  __shared__ int s_item, s_newk;
  W* slab = scratch + (size_t)blockIdx.x * slab_elems;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    const TsCore d = items[item];
    const int k = d.k;
    const W* Ra = tri + d.ra;
    const W* Rb = tri + d.rb;
    W* Rm = slab;
    W* Vm = Rm + (size_t)k * k;
    double* sig = reinterpret_cast<double*>(Vm + (size_t)k * k);
    int* ord = reinterpret_cast<int*>(sig + k);
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
      const int i = e % k, j = e / k;
      W s = zero<W>();
      for (int l = max(i, j); l < k; ++l) s = s + Ra[i + (size_t)l * k] * Rb[j + (size_t)l * k];
      Rm[e] = s;
    }
    __syncthreads();
    const bool conv = jacobi_svd(Rm, Vm, k, rs);
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      double s2 = 0.0;
      for (int i = 0; i < k; ++i) s2 += abs2(Rm[i + (size_t)j * k]);
      sig[j] = sqrt(s2);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      int r = 0;
      for (int i = 0; i < k; ++i) r += (sig[i] > sig[j]) || (sig[i] == sig[j] && i < j);
      ord[r] = j;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const double thr = sig[ord[0]] * eps;
      int nk = 0;
      while (nk < k && !(sig[ord[nk]] <= thr)) nk++;
      s_newk = nk;
    }
    __syncthreads();
    const int nk = s_newk;
    // Ma[i, c] = (Rb^T V[:, o])_i / sqrt(s_o), Mb[i, c] = (Ra^T conj(W[:, o]))_i / s_o^3/2
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
      const int i = e % k, c = e / k;
      W ma = zero<W>(), mb = zero<W>();
      if (c < nk) {
        const int o = ord[c];
        const double so = sig[o];
        for (int l = 0; l <= i; ++l) {
          ma = ma + Rb[l + (size_t)i * k] * Vm[l + (size_t)o * k];
          mb = mb + Ra[l + (size_t)i * k] * conjg(Rm[l + (size_t)o * k]);
        }
        const double rsq = 1.0 / sqrt(so);
        ma = scal(rsq, ma);
        mb = scal(rsq / so, mb);
      }
      maps[d.ma + e] = ma;
      maps[d.mb + e] = mb;
    }
    if (threadIdx.x == 0) {
      ranks[d.leaf] = nk;
      if (!conv && status[d.leaf] == kLeafOk) status[d.leaf] = kLeafSvdNoConverge;
    }
  }
}

// New factor columns of one segment: each thread takes rows, forms the k' outputs of a row
// (eight at a time, sums in increasing l) into the slab, then writes them over the row.
template <typename T, typename W>
__global__ void __launch_bounds__(kTruncThreads) tsapply_cta_kernel(const TsItem* __restrict__ items, int nitems,
                                                                     T* ws, const W* __restrict__ maps,
                                                                     const int* __restrict__ ranks, W* scratch,
                                                                     long long slab_elems, int* counter) {
  __shared__ int s_item;
  T* out = reinterpret_cast<T*>(scratch + (size_t)blockIdx.x * slab_elems);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    const TsItem d = items[item];
    const int k = d.k, nk = ranks[d.leaf], rows = d.rows;
    if (nk <= 0) continue;
    T* base = ws + d.src;
    const W* M = maps + d.map;
    for (int row = threadIdx.x; row < rows; row += blockDim.x) {
      for (int c0 = 0; c0 < nk; c0 += 8) {
        W acc[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = zero<W>();
        for (int l = 0; l < k; ++l) {
          const W a = widen(base[(size_t)l * d.ld + row]);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (c0 + q < nk) acc[q] = acc[q] + a * M[l + (size_t)(c0 + q) * k];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (c0 + q < nk) out[(size_t)(c0 + q) * rows + row] = narrow<T>(acc[q]);
      }
      // every input of this row is read: the outputs replace its first k' columns
      for (int c = 0; c < nk; ++c) base[(size_t)c * d.ld + row] = out[(size_t)c * rows + row];
    }
  }
}

}  // namespace

template <typename T>
long long truncate_slab_elems(int max_m, int max_n, int max_k) {
  long long k = max_k;
  // Wa, Wb, Ca, Cb, Ra, Rb, Rm, Vm, tau_a, tau_b, sigma (doubles), ord (ints) + slack
  return 2LL * (max_m + max_n) * k + 4 * k * k + 4 * k + 64;
}

template <typename T>
void launch_truncate(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, double epsilon, T* ws,
                     int* ranks, int* status, int* counter, typename Traits<T>::wide* scratch,
                     long long slab_elems, int grid, cudaStream_t s) {
  if (nleaves <= 0) return;
  int g = grid < nleaves ? grid : nleaves;
  truncate_kernel<T><<<g, kTruncThreads, 0, s>>>(d_leaves, d_order, nleaves, epsilon, ws, ranks, status, counter,
                                                scratch, slab_elems);
}

template <typename T>
void launch_unpack(const RkLeafDesc* d_leaves, int nleaves, const int* ranks, const RkStoreDesc* store,
                   const PanelDesc* panels, const T* arena, T* ws, cudaStream_t s) {
  if (nleaves <= 0) return;
  unpack_kernel<T><<<nleaves, 256, 0, s>>>(d_leaves, nleaves, ranks, store, panels, arena, ws);
}

template <typename T>
void launch_compact(const RkLeafDesc* d_leaves, int nleaves, const T* ws, const int* ranks,
                    const RkStoreDesc* store, const PanelDesc* panels, T* arena, cudaStream_t s) {
  if (nleaves <= 0) return;
  compact_kernel<T><<<nleaves, 256, 0, s>>>(d_leaves, nleaves, ws, ranks, store, panels, arena);
}

// HMAT_B200_TS_KMAX lowers the largest register-bucket rank (8, 16; tests use it to send
// leaves through the CTA-per-item phases).
template <typename T>
int ts_kmax() {
  int k = Traits<T>::is_complex ? 16 : 32;
  const char* s = getenv("HMAT_B200_TS_KMAX");
  if (s) {
    const int c = atoi(s);
    if (c >= 0 && c < k) k = c < 8 ? 0 : (c < 16 ? 8 : 16);
  }
  return k;
}
int ts_bucket(int k, int kmax) {
  if (k <= 0 || k > kmax) return 0;
  return k <= 8 ? 8 : (k <= 16 ? 16 : (k <= 24 ? 24 : 32));
}

// Grid of a warp-per-item launch: the resident CTAs of `kernel`, at most one warp per item.
template <typename F>
static int ts_grid(F kernel, int nitems, int warps = kTsWarps, size_t smem = 0) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, warps * 32, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int need = (nitems + warps - 1) / warps;
  const int g = persistent_grid(per_sm);
  return g < need ? g : need;
}

// Rows per lane of a tsqr chunk and of an apply chunk: the chunk is RPL x K wide scalars
// in each lane's registers.
template <typename W, int K>
struct TsShape {
  static constexpr int words = sizeof(W) / 8;
  // the chunk in registers: 64 doubles a lane (32 measured slower: twice the reductions
  // per row outweigh the extra resident warps)
  static constexpr int qr = 64 / (K * words) < 1 ? 1 : 64 / (K * words);
  static constexpr int ap = 32 / (K * words) < 1 ? 1 : 32 / (K * words);
  // warps per CTA of the core phase (the triangles of its 32 / K leaves sit in shared memory)
  static constexpr int core_warps = (32 / K) * K * K * words * 16 * 4 <= 40 * 1024 ? 4 : 2;
};

template <typename W, typename S, int K>
static void tsqr_run(const TsItem* items, int n, const S* src, W* tri, cudaStream_t s) {
  constexpr int RPL = TsShape<W, K>::qr;
  constexpr size_t per_warp = sizeof(TsqrSmem<W, S, K, RPL>);
  constexpr int NW = per_warp * 4 <= 64 * 1024 ? 4 : 2;
  constexpr size_t smem = per_warp * NW;
  auto kern = tsqr_kernel<W, S, K, RPL, NW>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  if (n <= 0) return;
  kern<<<ts_grid(kern, n, NW, smem), NW * 32, smem, s>>>(items, n, src, tri);
}

template <typename T, int K>
static void tsqr_k(const TsItem* items, int n, const T* ws, typename Traits<T>::wide* tri, bool from_tri,
                   cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  if (from_tri)
    tsqr_run<W, W, K>(items, n, tri, tri, s);
  else
    tsqr_run<W, T, K>(items, n, ws, tri, s);
}

template <typename T>
void launch_tsqr(int K, const TsItem* items, int nitems, const T* ws, typename Traits<T>::wide* tri,
                 bool from_tri, cudaStream_t s) {
  if (K == 8)
    tsqr_k<T, 8>(items, nitems, ws, tri, from_tri, s);
  else if (K == 16)
    tsqr_k<T, 16>(items, nitems, ws, tri, from_tri, s);
  else if constexpr (!Traits<T>::is_complex) {
    if (K == 24)
      tsqr_k<T, 24>(items, nitems, ws, tri, from_tri, s);
    else if (K == 32)
      tsqr_k<T, 32>(items, nitems, ws, tri, from_tri, s);
  }
}

template <typename T, int K>
static void tscore_k(const TsCore* items, int n, const typename Traits<T>::wide* tri,
                     typename Traits<T>::wide* maps, int* ranks, int* status, double eps, cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  constexpr int NW = TsShape<W, K>::core_warps;
  auto kern = tscore_kernel<W, K, NW>;
  if (n <= 0) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, kern);
    return;
  }
  kern<<<ts_grid(kern, n, NW), NW * 32, 0, s>>>(items, n, tri, maps, ranks, status, eps);
}

template <typename T>
void launch_tscore(int K, const TsCore* items, int nitems, const typename Traits<T>::wide* tri,
                   typename Traits<T>::wide* maps, int* ranks, int* status, double eps, cudaStream_t s) {
  if (K == 8)
    tscore_k<T, 8>(items, nitems, tri, maps, ranks, status, eps, s);
  else if (K == 16)
    tscore_k<T, 16>(items, nitems, tri, maps, ranks, status, eps, s);
  else if constexpr (!Traits<T>::is_complex) {
    if (K == 24)
      tscore_k<T, 24>(items, nitems, tri, maps, ranks, status, eps, s);
    else if (K == 32)
      tscore_k<T, 32>(items, nitems, tri, maps, ranks, status, eps, s);
  }
}

template <typename T, int K>
static void tsapply_k(const TsItem* items, int n, T* ws, const typename Traits<T>::wide* maps, const int* ranks,
                      cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  auto kern = tsapply_kernel<T, W, K, TsShape<W, K>::ap>;
  if (n <= 0) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, kern);
    return;
  }
  kern<<<ts_grid(kern, n), kTsWarps * 32, 0, s>>>(items, n, ws, maps, ranks);
}

template <typename T>
void launch_tsapply(int K, const TsItem* items, int nitems, T* ws, const typename Traits<T>::wide* maps,
                    const int* ranks, cudaStream_t s) {
  if (K == 8)
    tsapply_k<T, 8>(items, nitems, ws, maps, ranks, s);
  else if (K == 16)
    tsapply_k<T, 16>(items, nitems, ws, maps, ranks, s);
  else if constexpr (!Traits<T>::is_complex) {
    if (K == 24)
      tsapply_k<T, 24>(items, nitems, ws, maps, ranks, s);
    else if (K == 32)
      tsapply_k<T, 32>(items, nitems, ws, maps, ranks, s);
  }
}

// High-rank tall-skinny phases (tsqr_cta / tscore_cta / tsapply_cta), one launch each on a
// persistent grid of `grid` CTAs with a work counter (zeroed here, on the stream).
template <typename T>
void launch_tsqr_cta(const TsItem* items, int nitems, const T* ws, typename Traits<T>::wide* tri, bool from_tri,
                     typename Traits<T>::wide* scratch, long long slab, int grid, int* counter, cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  if (nitems <= 0) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, tsqr_cta_kernel<W, T>);
    cudaFuncGetAttributes(&a, tsqr_cta_kernel<W, W>);
    return;
  }
  cudaMemsetAsync(counter, 0, sizeof(int), s);
  const int g = grid < nitems ? grid : nitems;
  if (from_tri)
    tsqr_cta_kernel<W, W><<<g, kTruncThreads, 0, s>>>(items, nitems, tri, tri, scratch, slab, counter);
  else
    tsqr_cta_kernel<W, T><<<g, kTruncThreads, 0, s>>>(items, nitems, ws, tri, scratch, slab, counter);
}
template <typename T>
void launch_tscore_cta(const TsCore* items, int nitems, const typename Traits<T>::wide* tri,
                       typename Traits<T>::wide* maps, int* ranks, int* status, double eps,
                       typename Traits<T>::wide* scratch, long long slab, int grid, int* counter, cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  if (nitems <= 0) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, tscore_cta_kernel<W>);
    return;
  }
  cudaMemsetAsync(counter, 0, sizeof(int), s);
  const int g = grid < nitems ? grid : nitems;
  tscore_cta_kernel<W><<<g, kTruncThreads, 0, s>>>(items, nitems, tri, maps, ranks, status, eps, scratch, slab,
                                                   counter);
}
template <typename T>
void launch_tsapply_cta(const TsItem* items, int nitems, T* ws, const typename Traits<T>::wide* maps,
                        const int* ranks, typename Traits<T>::wide* scratch, long long slab, int grid, int* counter,
                        cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  if (nitems <= 0) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, tsapply_cta_kernel<T, W>);
    return;
  }
  cudaMemsetAsync(counter, 0, sizeof(int), s);
  const int g = grid < nitems ? grid : nitems;
  tsapply_cta_kernel<T, W><<<g, kTruncThreads, 0, s>>>(items, nitems, ws, maps, ranks, scratch, slab, counter);
}

// Loads every truncation kernel of the storage type T (the CUDA runtime otherwise loads a
// kernel at its first launch, inside the first assembly).
cudaError_t set_jacobi_max_sweeps(int sweeps) {
  const int v = sweeps < 1 ? 1 : sweeps;
  return cudaMemcpyToSymbol(g_jacobi_max_sweeps, &v, sizeof(int));
}

template <typename T>
void preload_truncate_kernels() {
  typedef typename Traits<T>::wide W;
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, truncate_kernel<T>);
  cudaFuncGetAttributes(&a, compact_kernel<T>);
  cudaFuncGetAttributes(&a, unpack_kernel<T>);
  const int kmax = ts_kmax<T>();
  for (int K : {8, 16, 24, 32}) {
    if (K > kmax) break;
    launch_tsqr<T>(K, nullptr, 0, nullptr, nullptr, false, 0);
    launch_tsqr<T>(K, nullptr, 0, nullptr, nullptr, true, 0);
    launch_tscore<T>(K, nullptr, 0, nullptr, nullptr, nullptr, nullptr, 0.0, 0);
    launch_tsapply<T>(K, nullptr, 0, nullptr, nullptr, nullptr, 0);
  }
  launch_tsqr_cta<T>(nullptr, 0, nullptr, nullptr, false, nullptr, 0, 0, nullptr, 0);
  launch_tscore_cta<T>(nullptr, 0, nullptr, nullptr, nullptr, nullptr, 0.0, nullptr, 0, 0, nullptr, 0);
  launch_tsapply_cta<T>(nullptr, 0, nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, 0);
}

#define HB_INST(T)                                                                                         \
  template long long truncate_slab_elems<T>(int, int, int);                                               \
  template void launch_truncate<T>(const RkLeafDesc*, const int*, int, double, T*, int*, int*, int*,     \
                                   typename Traits<T>::wide*, long long, int, cudaStream_t);               \
  template void launch_compact<T>(const RkLeafDesc*, int, const T*, const int*, const RkStoreDesc*,        \
                                  const PanelDesc*, T*, cudaStream_t);                                    \
  template void launch_unpack<T>(const RkLeafDesc*, int, const int*, const RkStoreDesc*, const PanelDesc*,  \
                                 const T*, T*, cudaStream_t);                                             \
  template void preload_truncate_kernels<T>();                                                            \
  template void launch_tsqr_cta<T>(const TsItem*, int, const T*, typename Traits<T>::wide*, bool,            \
                                   typename Traits<T>::wide*, long long, int, int*, cudaStream_t);         \
  template void launch_tscore_cta<T>(const TsCore*, int, const typename Traits<T>::wide*,                    \
                                     typename Traits<T>::wide*, int*, int*, double, typename Traits<T>::wide*, \
                                     long long, int, int*, cudaStream_t);                                  \
  template void launch_tsapply_cta<T>(const TsItem*, int, T*, const typename Traits<T>::wide*, const int*,   \
                                      typename Traits<T>::wide*, long long, int, int*, cudaStream_t);      \
  template int ts_kmax<T>();                                                                               \
  template void launch_tsqr<T>(int, const TsItem*, int, const T*, typename Traits<T>::wide*, bool,         \
                               cudaStream_t);                                                              \
  template void launch_tscore<T>(int, const TsCore*, int, const typename Traits<T>::wide*,                 \
                                 typename Traits<T>::wide*, int*, int*, double, cudaStream_t);             \
  template void launch_tsapply<T>(int, const TsItem*, int, T*, const typename Traits<T>::wide*, const int*, \
                                  cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
