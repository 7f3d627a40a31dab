// Batched ACA+ compression of admissible leaves, one CTA per leaf, persistent grid fed
// by a device work counter over leaves sorted by decreasing cost.
//
// The control flow is hmat-oss's doCompressionAcaPlus (compression.cpp:553-724) with its
// helpers findCol / findMinRow / findMinCol / updateRow / updateCol (compression.cpp:81-220)
// and the partial-ACA delegate doCompressionAcaPartial (compression.cpp:382-533), taken
// when cols * 100 < rows (compression.cpp:557-560).  Pivot selection keeps the BLAS
// i?amax rule (first index of the largest |x|, |Re|+|Im| for complex) and the
// strict-minimum / strict-maximum first-index rules of the scalar loops, so the FP64
// engine picks the reference's pivots.  Residual updates are per-element sequential in
// the rank index, each term rounded like the CPU axpy sequence they restate (see upd()).
//
// Vectors of a leaf live in its workspace slot (global memory, L1/L2 resident while the
// CTA works on it); FP64 accumulators carry the Frobenius-norm estimate for every T.
#include "block_reduce.cuh"
#include "kernels.h"

namespace hmatb200 {
namespace {

constexpr int kAcaSmallThreads = 64;
constexpr int kAcaThreads = 128;
constexpr int kAcaMidThreads = 256;
constexpr int kAcaBigThreads = 512;

template <typename T>
struct Aca {
  typedef typename Traits<T>::wide W;
  KernelParams kp;
  Points P;
  int row_off, m, col_off, n, kcap;
  T* A;  // m x kcap
  T* B;  // n x kcap
  T* aRef;
  T* bRef;
  unsigned char* rowFree;
  unsigned char* colFree;
  T* coef;  // shared [kcap]
  W* da;    // shared [kcap]
  W* db;    // shared [kcap]
  RedScratch* rs;

  __device__ T entry(int i, int j) const { return KernelEval<T>::eval(kp, P, row_off + i, col_off + j); }

  // out[e] = K(e) - sum_{l<k} coef[l] X[e, l] over len entries: each thread takes four
  // entries at a time (blockDim apart) and issues their factor loads together; every entry
  // is still updated in increasing l.
  template <typename F>
  __device__ void fill(F eval, const T* X, int len, int k, T* out) {
    constexpr int E = 4;
    const int nt = blockDim.x;
    for (int e0 = threadIdx.x; e0 < len; e0 += E * nt) {
      T v[E];
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = e0 + q * nt < len ? eval(e0 + q * nt) : zero<T>();
      int l = 0;
      for (; l + 4 <= k; l += 4) {
        T x[4][E];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int q = 0; q < E; ++q)
            x[u][q] = e0 + q * nt < len ? X[(size_t)(l + u) * len + e0 + q * nt] : zero<T>();
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int q = 0; q < E; ++q) v[q] = upd(coef[l + u], x[u][q], v[q]);
      }
      for (; l < k; ++l) {
#pragma unroll
        for (int q = 0; q < E; ++q)
          if (e0 + q * nt < len) v[q] = upd(coef[l], X[(size_t)l * len + e0 + q * nt], v[q]);
      }
#pragma unroll
      for (int q = 0; q < E; ++q)
        if (e0 + q * nt < len) out[e0 + q * nt] = v[q];
    }
  }
  // out[j] = K(i, j) - sum_{l<k} A[i, l] B[j, l]   (getRow + updateRow)
  __device__ void fill_row(int i, int k, T* out) {
    __syncthreads();
    for (int l = threadIdx.x; l < k; l += blockDim.x) coef[l] = -A[(size_t)l * m + i];
    __syncthreads();
    fill([&](int j) { return entry(i, j); }, B, n, k, out);
    __syncthreads();
  }
  // out[i] = K(i, j) - sum_{l<k} B[j, l] A[i, l]   (getCol + updateCol)
  __device__ void fill_col(int j, int k, T* out) {
    __syncthreads();
    for (int l = threadIdx.x; l < k; l += blockDim.x) coef[l] = -B[(size_t)l * n + j];
    __syncthreads();
    fill([&](int i) { return entry(i, j); }, A, m, k, out);
    __syncthreads();
  }
  __device__ void scale(T* v, int len, T s) {
    for (int e = threadIdx.x; e < len; e += blockDim.x) v[e] = mul_rn(v[e], s);
    __syncthreads();
  }
  // v += a * x
  __device__ void axpy(T a, const T* x, T* v, int len) {
    for (int e = threadIdx.x; e < len; e += blockDim.x) v[e] = upd(a, x[e], v[e]);
    __syncthreads();
  }
  __device__ bool is_zero(const T* v, int len) {
    bool nz = false;
    for (int e = threadIdx.x; e < len; e += blockDim.x) nz |= !is_zero_val(v[e]);
    return !block_any(nz, *rs);
  }
  __device__ int iamax(const T* v, int len) {
    KeyIdx b{-1.0, -1};
    for (int e = threadIdx.x; e < len; e += blockDim.x) {
      double kk = amax_key(v[e]);
      if (kk > b.key) { b.key = kk; b.idx = e; }
    }
    return block_arg<true>(b, *rs).idx;
  }
  // first index of the strict minimum of |v|^2 over free entries (DBL_MAX start)
  __device__ int argmin_free(const T* v, const unsigned char* fr, int len) {
    KeyIdx b{DBL_MAX, -1};
    for (int e = threadIdx.x; e < len; e += blockDim.x) {
      if (fr[e]) {
        double kk = abs2(v[e]);
        if (kk < b.key) { b.key = kk; b.idx = e; }
      }
    }
    return block_arg<false>(b, *rs).idx;
  }
  // first index of the strict maximum of |v|^2 over free entries (0 start), -1 if none
  __device__ int argmax_free_pos(const T* v, const unsigned char* fr, int len) {
    KeyIdx b{0.0, -1};
    for (int e = threadIdx.x; e < len; e += blockDim.x) {
      if (fr[e]) {
        double kk = abs2(v[e]);
        if (kk > b.key) { b.key = kk; b.idx = e; }
      }
    }
    return block_arg<true>(b, *rs).idx;
  }
  __device__ void clear_flag(unsigned char* fr, int idx) {
    __syncthreads();
    if (threadIdx.x == 0) fr[idx] = 0;
    __syncthreads();
  }

  // findCol: first free column that is not identically zero (raw, not updated)
  __device__ int find_col(T* out) {
    for (int j = 0; j < n; ++j) {
      if (colFree[j]) {
        fill_col(j, 0, out);
        clear_flag(colFree, j);
        if (!is_zero(out, m)) return j;
      }
    }
    return -1;
  }
  __device__ int find_min_row(int k, const T* ref, T* out) {
    for (;;) {
      int i = argmin_free(ref, rowFree, m);
      if (i < 0) return -1;
      fill_row(i, k, out);
      clear_flag(rowFree, i);
      if (!is_zero(out, n)) return i;
    }
  }
  __device__ int find_min_col(int k, const T* ref, T* out) {
    for (;;) {
      int j = argmin_free(ref, colFree, n);
      if (j < 0) return -1;
      fill_col(j, k, out);
      clear_flag(colFree, j);
      if (!is_zero(out, m)) return j;
    }
  }

  // Gram terms of the new pair (a_k, b_k) against the previous ones, in FP64:
  // returns ||a_k||^2 ||b_k||^2 and adds 2 sum_l Re(<a_k,a_l><b_k,b_l>) + that to est.
  __device__ double update_estimate(int k, double& est) {
    const T* a = A + (size_t)k * m;
    const T* b = B + (size_t)k * n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __shared__ double s_norm[2];
    for (int t = warp; t < 2 * k + 2; t += nw) {
      const bool isA = (t < k) || (t == 2 * k);
      const T* x = isA ? a : b;
      const T* y = t < k ? A + (size_t)t * m : (t < 2 * k ? B + (size_t)(t - k) * n : x);
      const int len = isA ? m : n;
      W acc = zero<W>();
      for (int e = lane; e < len; e += 32) acc = acc + widen(conjg(x[e])) * widen(y[e]);
      acc = warp_sum(acc);
      if (lane == 0) {
        if (t < k) da[t] = acc;
        else if (t < 2 * k) db[t - k] = acc;
        else s_norm[t - 2 * k] = real_part(acc);
      }
    }
    __syncthreads();
    double ne = 0.0;
    for (int l = 0; l < k; ++l) ne += real_part(da[l] * db[l]);
    est += 2.0 * ne;
    double ab = s_norm[0] * s_norm[1];
    est += ab;
    __syncthreads();
    return ab;
  }

  __device__ void init_flags() {
    for (int e = threadIdx.x; e < m; e += blockDim.x) rowFree[e] = 1;
    for (int e = threadIdx.x; e < n; e += blockDim.x) colFree[e] = 1;
    __syncthreads();
  }

  // doCompressionAcaPartial, no random pivots.  Returns the rank; sets *overflow when the
  // slot capacity is reached first.
  __device__ int partial(double eps, bool* overflow) {
    const int maxK = min(m, n);
    init_flags();
    double est = 0.0;
    int row_index = 0, J = 0, k = 0, rowPivotCount = 0;
    do {
      if (k >= kcap) { *overflow = true; break; }
      T* bCol = B + (size_t)k * n;
      fill_row(row_index, k, bCol);
      clear_flag(rowFree, row_index);
      int jj = argmax_free_pos(bCol, colFree, n);
      if (jj >= 0) J = jj;
      T bj = bCol[J];
      if (is_zero_val(bj)) {
        row_index = 0;
        while (row_index < m && !rowFree[row_index]) row_index++;
      } else {
        scale(bCol, n, recip(bj));
        T* aCol = A + (size_t)k * m;
        fill_col(J, k, aCol);
        clear_flag(colFree, J);
        int ii = argmax_free_pos(aCol, rowFree, m);
        if (ii >= 0) row_index = ii;
        double ab = update_estimate(k, est);
        k++;
        if (ab < eps * eps * est) break;
      }
      rowPivotCount++;
    } while (rowPivotCount < maxK && row_index < m);
    return k;
  }

  // doCompressionAcaPlus.
  __device__ int plus(double eps, bool* overflow) {
    const int maxK = min(m, n);
    init_flags();
    double est = 0.0;
    int k = 0;
    int j_ref = find_col(aRef);
    if (j_ref < 0) return 0;
    int i_ref = find_min_row(0, aRef, bRef);
    if (i_ref < 0) return 0;  // cannot happen once a non-zero column exists; keeps indices valid
    do {
      if (k >= kcap) { *overflow = true; break; }
      T* aVec = A + (size_t)k * m;
      T* bVec = B + (size_t)k * n;
      KeyIdx ka{-1.0, -1}, kb{-1.0, -1};
      for (int e = threadIdx.x; e < m; e += blockDim.x) {
        double kk = amax_key(aRef[e]);
        if (kk > ka.key) { ka.key = kk; ka.idx = e; }
      }
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        double kk = amax_key(bRef[e]);
        if (kk > kb.key) { kb.key = kk; kb.idx = e; }
      }
      block_argmax2(ka, kb, *rs);
      int i_star = ka.idx, j_star = kb.idx;
      if (abs2(aRef[i_star]) > abs2(bRef[j_star])) {
        fill_row(i_star, k, bVec);
        j_star = iamax(bVec, n);
        T pivot = bVec[j_star];
        fill_col(j_star, k, aVec);
        if (!is_zero_val(pivot)) scale(aVec, m, recip(pivot));
      } else {
        fill_col(j_star, k, aVec);
        i_star = iamax(aVec, m);
        T pivot = aVec[i_star];
        fill_row(i_star, k, bVec);
        if (!is_zero_val(pivot)) scale(bVec, n, recip(pivot));
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        rowFree[i_star] = 0;
        colFree[j_star] = 0;
      }
      double ab = update_estimate(k, est);
      k++;
      if (ab < eps * eps * est) break;

      // aRef -= b_k[j_ref] a_k ; bRef -= a_k[i_ref] b_k
      T ca = -bVec[j_ref];
      T cb = -aVec[i_ref];
      axpy(ca, aVec, aRef, m);
      axpy(cb, bVec, bRef, n);
      const bool needNewA = (j_star == j_ref) || is_zero(aRef, m);
      const bool needNewB = (i_star == i_ref) || is_zero(bRef, n);
      if (needNewA && needNewB) {
        bool found = false;
        while (!found) {
          j_ref = find_col(aRef);
          if (j_ref < 0) break;
          fill_col(j_ref, k, aRef);
          found = !is_zero(aRef, m);
        }
        if (!found) break;
        i_ref = find_min_row(k, aRef, bRef);
        if (i_ref < 0) break;
      } else if (needNewB) {
        i_ref = find_min_row(k, aRef, bRef);
        if (i_ref < 0) break;
      } else if (needNewA) {
        j_ref = find_min_col(k, bRef, aRef);
        if (j_ref < 0) break;
      }
    } while (k < maxK);
    return k;
  }
};

template <typename T, int NT>
__global__ void __launch_bounds__(NT) aca_kernel(const RkLeafDesc* __restrict__ leaves,
                                                          const int* __restrict__ order, int nleaves,
                                                          KernelParams kp, Points pts, double eps, T* ws,
                                                          unsigned char* flags, int* ranks, int* status,
                                                          int* counter, int kcap_max) {
  typedef typename Traits<T>::wide W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  W* da = reinterpret_cast<W*>(smem_raw);
  W* db = da + kcap_max;
  T* coef = reinterpret_cast<T*>(db + kcap_max);
  __shared__ RedScratch rs;
  __shared__ int s_item;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nleaves) break;
    const int leaf = order[item];
    const RkLeafDesc d = leaves[leaf];
    Aca<T> c;
    c.kp = kp;
    c.P = pts;
    c.row_off = d.row_off;
    c.m = d.m;
    c.col_off = d.col_off;
    c.n = d.n;
    c.kcap = d.kcap;
    T* slot = ws + d.ws_off;
    c.A = slot;
    c.B = slot + (size_t)d.m * d.kcap;
    c.aRef = c.B + (size_t)d.n * d.kcap;
    c.bRef = c.aRef + d.m;
    c.rowFree = flags + d.fl_off;
    c.colFree = c.rowFree + d.m;
    c.coef = coef;
    c.da = da;
    c.db = db;
    c.rs = &rs;
    bool overflow = false;
    int k;
    if (d.n * 100 < d.m) k = c.partial(eps, &overflow);
    else k = c.plus(eps, &overflow);
    if (threadIdx.x == 0) {
      ranks[leaf] = k;
      status[leaf] = overflow ? kLeafAcaCapacity : kLeafOk;
    }
  }
}

// ---------------------------------------------------------------------------------
// Warp-per-leaf ACA+ for small leaves (m, n <= 64, the plus path): the control flow, pivot
// rules and per-element arithmetic of Aca::plus, run by one warp without block barriers.
// Lane l owns rows l and l + 32 of the new column and of the reference column, and columns
// l and l + 32 of the new row and of the reference row; the factors grow in the warp's
// shared memory (column-major, kAwLen rows a column) and go to the slot at the end.  The
// free-row / free-column flags are 64-bit masks held by every lane.  Pivot searches keep
// the first-index rules, and the FP64 Gram terms are summed per lane over rows lane,
// lane + 32 and then by warp_sum, as in the CTA kernel, so both kernels build the same
// factors.
constexpr int kAwWarps = 4;
constexpr int kAwLen = 64;

__device__ inline float aw_shfl(float v, int s) { return __shfl_sync(0xffffffffu, v, s); }
__device__ inline double aw_shfl(double v, int s) { return __shfl_sync(0xffffffffu, v, s); }
__device__ inline cfloat aw_shfl(cfloat v, int s) {
  return cfloat{__shfl_sync(0xffffffffu, v.x, s), __shfl_sync(0xffffffffu, v.y, s)};
}
__device__ inline cdouble aw_shfl(cdouble v, int s) {
  return cdouble{__shfl_sync(0xffffffffu, v.x, s), __shfl_sync(0xffffffffu, v.y, s)};
}
__device__ inline unsigned long long aw_mask(int len) { return len >= 64 ? ~0ull : ((1ull << len) - 1ull); }

template <typename T>
struct AcaWarp {
  typedef typename Traits<T>::wide W;
  KernelParams kp;
  Points P;
  int row_off, m, col_off, n, kc;
  T* sA;  // [kc][kAwLen]
  T* sB;  // [kc][kAwLen]
  unsigned long long rowFree, colFree;
  int lane;

  __device__ T entry(int i, int j) const { return KernelEval<T>::eval(kp, P, row_off + i, col_off + j); }
  // element idx of a lane-distributed vector, in every lane
  __device__ T get(const T (&v)[2], int idx) const {
    const T mine = (idx >> 5) ? v[1] : v[0];
    return aw_shfl(mine, idx & 31);
  }
  // out = K(i, :) - sum_{l<k} A[i, l] B[:, l]   (getRow + updateRow)
  __device__ void fill_row(int i, int k, T (&out)[2]) const {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int j = lane + 32 * r;
      T v = zero<T>();
      if (j < n) {
        v = entry(i, j);
        for (int l = 0; l < k; ++l) v = upd(-sA[l * kAwLen + i], sB[l * kAwLen + j], v);
      }
      out[r] = v;
    }
  }
  // out = K(:, j) - sum_{l<k} B[j, l] A[:, l]   (getCol + updateCol)
  __device__ void fill_col(int j, int k, T (&out)[2]) const {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int i = lane + 32 * r;
      T v = zero<T>();
      if (i < m) {
        v = entry(i, j);
        for (int l = 0; l < k; ++l) v = upd(-sB[l * kAwLen + j], sA[l * kAwLen + i], v);
      }
      out[r] = v;
    }
  }
  __device__ bool nonzero(const T (&v)[2], int len) const {
    const bool nz = (lane < len && !is_zero_val(v[0])) || (lane + 32 < len && !is_zero_val(v[1]));
    return __any_sync(0xffffffffu, nz);
  }
  __device__ int bcast_idx(KeyIdx b) const { return __shfl_sync(0xffffffffu, b.idx, 0); }
  __device__ int iamax(const T (&v)[2], int len) const {
    KeyIdx b{-1.0, -1};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = lane + 32 * r;
      if (e < len) {
        const double kk = amax_key(v[r]);
        if (kk > b.key) {
          b.key = kk;
          b.idx = e;
        }
      }
    }
    return bcast_idx(warp_arg<true>(b));
  }
  // first index of the strict minimum of |v|^2 over free entries (DBL_MAX start)
  __device__ int argmin_free(const T (&v)[2], unsigned long long fr, int len) const {
    KeyIdx b{DBL_MAX, -1};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = lane + 32 * r;
      if (e < len && ((fr >> e) & 1ull)) {
        const double kk = abs2(v[r]);
        if (kk < b.key) {
          b.key = kk;
          b.idx = e;
        }
      }
    }
    return bcast_idx(warp_arg<false>(b));
  }
  __device__ int find_col(T (&out)[2]) {
    for (int j = 0; j < n; ++j) {
      if ((colFree >> j) & 1ull) {
        fill_col(j, 0, out);
        colFree &= ~(1ull << j);
        if (nonzero(out, m)) return j;
      }
    }
    return -1;
  }
  __device__ int find_min_row(int k, const T (&ref)[2], T (&out)[2]) {
    for (;;) {
      const int i = argmin_free(ref, rowFree, m);
      if (i < 0) return -1;
      fill_row(i, k, out);
      rowFree &= ~(1ull << i);
      if (nonzero(out, n)) return i;
    }
  }
  __device__ int find_min_col(int k, const T (&ref)[2], T (&out)[2]) {
    for (;;) {
      const int j = argmin_free(ref, colFree, n);
      if (j < 0) return -1;
      fill_col(j, k, out);
      colFree &= ~(1ull << j);
      if (nonzero(out, m)) return j;
    }
  }
  // <x, y> over len entries of two stored columns: per-lane rows lane, lane + 32, then warp_sum
  __device__ W dot(const T* x, const T* y, int len) const {
    W acc = zero<W>();
    for (int e = lane; e < len; e += 32) acc = acc + widen(conjg(x[e])) * widen(y[e]);
    return warp_bcast(warp_sum(acc));
  }
  // Gram terms of the new pair (a_k, b_k), as Aca::update_estimate.
  __device__ double update_estimate(int k, double& est) const {
    const T* a = sA + k * kAwLen;
    const T* b = sB + k * kAwLen;
    double ne = 0.0;
    for (int l = 0; l < k; ++l) {
      const W da = dot(a, sA + l * kAwLen, m);
      const W db = dot(b, sB + l * kAwLen, n);
      ne += real_part(da * db);
    }
    const double na = real_part(dot(a, a, m)), nb = real_part(dot(b, b, n));
    est += 2.0 * ne;
    const double ab = na * nb;
    est += ab;
    return ab;
  }
  __device__ void store(T* col, const T (&v)[2], int len) const {
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (lane + 32 * r < len) col[lane + 32 * r] = v[r];
  }

  __device__ int plus(double eps, bool* overflow) {
    const int maxK = min(m, n);
    rowFree = aw_mask(m);
    colFree = aw_mask(n);
    T aRef[2], bRef[2];
    double est = 0.0;
    int k = 0;
    int j_ref = find_col(aRef);
    if (j_ref < 0) return 0;
    int i_ref = find_min_row(0, aRef, bRef);
    if (i_ref < 0) return 0;
    do {
      if (k >= kc) {
        *overflow = true;
        break;
      }
      int i_star = iamax(aRef, m), j_star = iamax(bRef, n);
      if (i_star < 0 || j_star < 0) break;  // no ordered entry (NaN data): stop, never index with -1
      T aVec[2], bVec[2];
      if (abs2(get(aRef, i_star)) > abs2(get(bRef, j_star))) {
        fill_row(i_star, k, bVec);
        j_star = iamax(bVec, n);
        if (j_star < 0) break;
        const T pivot = get(bVec, j_star);
        fill_col(j_star, k, aVec);
        if (!is_zero_val(pivot)) {
          const T s = recip(pivot);
          aVec[0] = mul_rn(aVec[0], s);
          aVec[1] = mul_rn(aVec[1], s);
        }
      } else {
        fill_col(j_star, k, aVec);
        i_star = iamax(aVec, m);
        if (i_star < 0) break;
        const T pivot = get(aVec, i_star);
        fill_row(i_star, k, bVec);
        if (!is_zero_val(pivot)) {
          const T s = recip(pivot);
          bVec[0] = mul_rn(bVec[0], s);
          bVec[1] = mul_rn(bVec[1], s);
        }
      }
      store(sA + k * kAwLen, aVec, m);
      store(sB + k * kAwLen, bVec, n);
      __syncwarp();
      rowFree &= ~(1ull << i_star);
      colFree &= ~(1ull << j_star);
      const double ab = update_estimate(k, est);
      k++;
      if (ab < eps * eps * est) break;

      // aRef -= b_k[j_ref] a_k ; bRef -= a_k[i_ref] b_k
      const T ca = -get(bVec, j_ref);
      const T cb = -get(aVec, i_ref);
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        if (lane + 32 * r < m) aRef[r] = upd(ca, aVec[r], aRef[r]);
        if (lane + 32 * r < n) bRef[r] = upd(cb, bVec[r], bRef[r]);
      }
      const bool needNewA = (j_star == j_ref) || !nonzero(aRef, m);
      const bool needNewB = (i_star == i_ref) || !nonzero(bRef, n);
      if (needNewA && needNewB) {
        bool found = false;
        while (!found) {
          j_ref = find_col(aRef);
          if (j_ref < 0) break;
          fill_col(j_ref, k, aRef);
          found = nonzero(aRef, m);
        }
        if (!found) break;
        i_ref = find_min_row(k, aRef, bRef);
        if (i_ref < 0) break;
      } else if (needNewB) {
        i_ref = find_min_row(k, aRef, bRef);
        if (i_ref < 0) break;
      } else if (needNewA) {
        j_ref = find_min_col(k, bRef, aRef);
        if (j_ref < 0) break;
      }
    } while (k < maxK);
    return k;
  }
};

template <typename T>
__global__ void __launch_bounds__(kAwWarps * 32) aca_warp_kernel(const RkLeafDesc* __restrict__ leaves,
                                                                 const int* __restrict__ order, int nleaves,
                                                                 KernelParams kp, Points pts, double eps, T* ws,
                                                                 int* ranks, int* status, int* counter, int kc) {
  extern __shared__ __align__(16) unsigned char aw_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* sA = reinterpret_cast<T*>(aw_smem) + (size_t)warp * 2 * kc * kAwLen;
  T* sB = sA + (size_t)kc * kAwLen;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nleaves) break;
    const int leaf = order[item];
    const RkLeafDesc d = leaves[leaf];
    AcaWarp<T> c;
    c.kp = kp;
    c.P = pts;
    c.row_off = d.row_off;
    c.m = d.m;
    c.col_off = d.col_off;
    c.n = d.n;
    c.kc = min(d.kcap, kc);
    c.sA = sA;
    c.sB = sB;
    c.lane = lane;
    bool overflow = false;
    __syncwarp();
    const int k = c.plus(eps, &overflow);
    __syncwarp();
    T* A = ws + d.ws_off;
    T* B = A + (size_t)d.m * d.kcap;
    for (int l = 0; l < k; ++l) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int e = lane + 32 * r;
        if (e < d.m) A[(size_t)l * d.m + e] = sA[l * kAwLen + e];
        if (e < d.n) B[(size_t)l * d.n + e] = sB[l * kAwLen + e];
      }
    }
    if (lane == 0) {
      ranks[leaf] = k;
      status[leaf] = overflow ? kLeafAcaCapacity : kLeafOk;
    }
  }
}

// Dense-SVD compression of small admissible blocks (doCompressionSVD, compression.cpp:241-251):
// the block M is written into the slot as a trivially exact factorisation M = A B^T
// (A = M, B = I when m >= n; A = I, B = M^T otherwise, rank min(m, n)), so the truncation
// phase, whose core is the SVD of Ra Rb^T, computes the truncated SVD of M.
template <typename T>
__global__ void dense_to_rk_kernel(const RkLeafDesc* __restrict__ leaves, const int* __restrict__ order,
                                   int nleaves, KernelParams kp, Points pts, T* ws, int* ranks, int* status) {
  const int item = blockIdx.x;
  if (item >= nleaves) return;
  const int leaf = order[item];
  const RkLeafDesc d = leaves[leaf];
  const int m = d.m, n = d.n, k = min(m, n);
  T* A = ws + d.ws_off;
  T* B = A + (size_t)m * d.kcap;
  if (d.kcap < k) {
    if (threadIdx.x == 0) {
      ranks[leaf] = 0;
      status[leaf] = kLeafBadShape;
    }
    return;
  }
  for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
    const int i = e % m, j = e / m;
    // a multi-strata kernel: the sum of its strata (the SVD compression is not incremental)
    const T v = kp.nstrata > 0 ? KernelEval<T>::eval_sum(kp, pts, d.row_off + i, d.col_off + j)
                               : KernelEval<T>::eval(kp, pts, d.row_off + i, d.col_off + j);
    if (m >= n) A[(size_t)j * m + i] = v;  // A = M (m x n)
    else B[(size_t)i * n + j] = v;         // B = M^T (n x m)
  }
  if (m >= n) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) B[e] = (e % (n + 1) == 0) ? one<T>() : zero<T>();
  } else {
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] = (e % (m + 1) == 0) ? one<T>() : zero<T>();
  }
  if (threadIdx.x == 0) {
    ranks[leaf] = k;
    status[leaf] = kLeafOk;
  }
}

}  // namespace

template <typename T>
void launch_dense_to_rk(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp,
                        Points pts, T* ws, int* ranks, int* status, cudaStream_t s) {
  if (nleaves <= 0) return;
  dense_to_rk_kernel<T><<<nleaves, 256, 0, s>>>(d_leaves, d_order, nleaves, kp, pts, ws, ranks, status);
}

int persistent_grid(int blocks_per_sm) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms * blocks_per_sm;
}

template <typename T, int NT>
static void aca_run(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp, Points pts,
                    double epsilon, T* ws, unsigned char* flags, int* ranks, int* status, int* counter, int kcap_max,
                    int grid, cudaStream_t s) {
  typedef typename Traits<T>::wide W;
  size_t smem = (size_t)kcap_max * (2 * sizeof(W) + sizeof(T));
  if (smem > 48 * 1024) cudaFuncSetAttribute(aca_kernel<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int g = grid < nleaves ? grid : nleaves;
  aca_kernel<T, NT><<<g, NT, smem, s>>>(d_leaves, d_order, nleaves, kp, pts, epsilon, ws, flags, ranks, status,
                                        counter, kcap_max);
}

template <typename T>
void launch_aca(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp, Points pts,
                double epsilon, T* ws, unsigned char* flags, int* ranks, int* status, int* counter, int kcap_max,
                int grid, cudaStream_t s, int threads) {
  if (nleaves <= 0) return;
  if (threads >= kAcaBigThreads)
    aca_run<T, kAcaBigThreads>(d_leaves, d_order, nleaves, kp, pts, epsilon, ws, flags, ranks, status, counter,
                               kcap_max, grid, s);
  else if (threads >= kAcaMidThreads)
    aca_run<T, kAcaMidThreads>(d_leaves, d_order, nleaves, kp, pts, epsilon, ws, flags, ranks, status, counter,
                               kcap_max, grid, s);
  else if (threads <= kAcaSmallThreads)
    aca_run<T, kAcaSmallThreads>(d_leaves, d_order, nleaves, kp, pts, epsilon, ws, flags, ranks, status, counter,
                                 kcap_max, grid, s);
  else
    aca_run<T, kAcaThreads>(d_leaves, d_order, nleaves, kp, pts, epsilon, ws, flags, ranks, status, counter,
                            kcap_max, grid, s);
}

template <typename T, int NT>
static int aca_resident_per_sm(int kcap_max) {
  typedef typename Traits<T>::wide W;
  const size_t smem = (size_t)kcap_max * (2 * sizeof(W) + sizeof(T));
  if (smem > 48 * 1024) cudaFuncSetAttribute(aca_kernel<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, aca_kernel<T, NT>, NT, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return per_sm;
}

// Rank capacity of the warp-per-leaf kernel's shared factors (its slots are 2 x 64 x kc
// scalars a warp).
template <typename T>
int aca_warp_cap() {
  return sizeof(T) <= 4 ? 32 : (sizeof(T) <= 8 ? 24 : 16);
}
bool aca_warp_eligible(int m, int n) { return m <= kAwLen && n <= kAwLen && !(n * 100 < m); }

template <typename T>
void launch_aca_warp(const RkLeafDesc* d_leaves, const int* d_order, int nleaves, const KernelParams& kp,
                     Points pts, double epsilon, T* ws, int* ranks, int* status, int* counter, int kcap_max,
                     cudaStream_t s) {
  const int kc = kcap_max < aca_warp_cap<T>() ? kcap_max : aca_warp_cap<T>();
  const size_t smem = (size_t)kAwWarps * 2 * kc * kAwLen * sizeof(T);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(aca_warp_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kAwWarps * 2 * aca_warp_cap<T>() * kAwLen * sizeof(T)));
    attr = true;
  }
  if (nleaves <= 0) return;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, aca_warp_kernel<T>, kAwWarps * 32, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int g = persistent_grid(per_sm);
  const int need = (nleaves + kAwWarps - 1) / kAwWarps;
  if (g > need) g = need;
  aca_warp_kernel<T><<<g, kAwWarps * 32, smem, s>>>(d_leaves, d_order, nleaves, kp, pts, epsilon, ws, ranks,
                                                    status, counter, kc);
}

template <typename T>
int aca_concurrency(int threads, int kcap_max) {
  if (threads == 0) {
    const int kc = kcap_max < aca_warp_cap<T>() ? kcap_max : aca_warp_cap<T>();
    const size_t smem = (size_t)kAwWarps * 2 * kc * kAwLen * sizeof(T);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, aca_warp_kernel<T>, kAwWarps * 32, smem) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    return persistent_grid(per_sm) * kAwWarps;
  }
  if (threads >= kAcaBigThreads) return persistent_grid(aca_resident_per_sm<T, kAcaBigThreads>(kcap_max));
  if (threads >= kAcaMidThreads) return persistent_grid(aca_resident_per_sm<T, kAcaMidThreads>(kcap_max));
  if (threads <= kAcaSmallThreads) return persistent_grid(aca_resident_per_sm<T, kAcaSmallThreads>(kcap_max));
  return persistent_grid(aca_resident_per_sm<T, kAcaThreads>(kcap_max));
}

template <typename T>
void preload_aca_kernels() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, aca_kernel<T, kAcaSmallThreads>);
  cudaFuncGetAttributes(&a, aca_kernel<T, kAcaThreads>);
  cudaFuncGetAttributes(&a, aca_kernel<T, kAcaMidThreads>);
  cudaFuncGetAttributes(&a, aca_kernel<T, kAcaBigThreads>);
  cudaFuncGetAttributes(&a, dense_to_rk_kernel<T>);
  launch_aca_warp<T>(nullptr, nullptr, 0, KernelParams{}, Points{}, 0.0, nullptr, nullptr, nullptr, nullptr, 1, 0);
}

#define HB_INST(T)                                                                                           \
  template void preload_aca_kernels<T>();                                                                  \
  template int aca_concurrency<T>(int, int);                                                               \
  template void launch_aca_warp<T>(const RkLeafDesc*, const int*, int, const KernelParams&, Points, double, T*, \
                                   int*, int*, int*, int, cudaStream_t);                                    \
  template void launch_aca<T>(const RkLeafDesc*, const int*, int, const KernelParams&, Points, double, T*, \
                              unsigned char*, int*, int*, int*, int, int, cudaStream_t, int);               \
  template void launch_dense_to_rk<T>(const RkLeafDesc*, const int*, int, const KernelParams&, Points, T*, \
                                      int*, int*, cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
