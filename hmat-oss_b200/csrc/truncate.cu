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
#include "block_reduce.cuh"
#include "kernels.h"

namespace hmatb200 {
namespace {

constexpr int kTruncThreads = 256;
constexpr int kJacobiMaxSweeps = 60;

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
  __shared__ int s_rot;
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
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

// Writes A as row panels (len x k column-major each) and B transposed (k x n column-major).
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
  for (int e = threadIdx.x; e < d.n * k; e += blockDim.x) {
    const int l = e % k, j = e / k;
    bt[e] = B[(size_t)l * d.n + j];
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
void launch_compact(const RkLeafDesc* d_leaves, int nleaves, const T* ws, const int* ranks,
                    const RkStoreDesc* store, const PanelDesc* panels, T* arena, cudaStream_t s) {
  if (nleaves <= 0) return;
  compact_kernel<T><<<nleaves, 256, 0, s>>>(d_leaves, nleaves, ws, ranks, store, panels, arena);
}

#define HB_INST(T)                                                                                         \
  template long long truncate_slab_elems<T>(int, int, int);                                               \
  template void launch_truncate<T>(const RkLeafDesc*, const int*, int, double, T*, int*, int*, int*,     \
                                   typename Traits<T>::wide*, long long, int, cudaStream_t);               \
  template void launch_compact<T>(const RkLeafDesc*, int, const T*, const int*, const RkStoreDesc*,        \
                                  const PanelDesc*, T*, cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
