// Multi-strata assembly on the device: the steps that join a further stratum to the factors a
// leaf already holds.  Restates the loop of compress() over strata (compression.cpp:745-773):
// after stratum 0 (ACA+ and truncation), each further stratum's ACA+ factors A_s B_s^T are
// added by RkMatrix::axpy with a negative epsilon, that is formattedAddParts without its own
// truncation (rk_matrix.cpp:846-983), then the sum is truncated:
//   summed rank < min(m, n)   concatenation [A | A_s], [B | B_s]                (append_kernel)
//   otherwise                 the full block A B^T + A_s B_s^T compressed by SVD
//                             (rk_matrix.cpp:985-1009), written here as its exact
//                             factorisation D I^T or I D^T for the dense-SVD phase
//                             (exact_kernel)
// The ACA of stratum s runs on the plain kernel with the stratum's parameter; its weight w_s
// multiplies the A factor when it is joined (scale_a_kernel for stratum 0).
#include "kernels.h"

namespace hmatb200 {
namespace {

__device__ inline float scale_by(float v, double w) { return (float)w * v; }
__device__ inline double scale_by(double v, double w) { return __dmul_rn(w, v); }
__device__ inline cfloat scale_by(cfloat v, double w) { return cfloat{(float)w * v.x, (float)w * v.y}; }
__device__ inline cdouble scale_by(cdouble v, double w) { return cdouble{__dmul_rn(w, v.x), __dmul_rn(w, v.y)}; }

// A[:, 0 .. rank) *= w for the slots of the leaves in `order`.
template <typename T>
__global__ void __launch_bounds__(256) scale_a_kernel(const RkLeafDesc* __restrict__ leaves,
                                                      const int* __restrict__ order, int count,
                                                      const int* __restrict__ ranks, double w, T* ws) {
  const int item = blockIdx.x;
  if (item >= count) return;
  const int b = order[item];
  const RkLeafDesc d = leaves[b];
  T* A = ws + d.ws_off;
  const long long n = (long long)d.m * ranks[b];
  for (long long e = threadIdx.x; e < n; e += blockDim.x) A[e] = scale_by(A[e], w);
}

// Slot b of `dst` gets, after the kcur[b] columns already unpacked there, the ks[b] columns of
// the stratum's factors from slot b of `src`: A_s scaled by w, B_s as it is.
template <typename T>
__global__ void __launch_bounds__(256) append_kernel(const RkLeafDesc* __restrict__ src_desc,
                                                     const RkLeafDesc* __restrict__ dst_desc, int nb,
                                                     const int* __restrict__ kcur, const int* __restrict__ ks,
                                                     double w, const T* __restrict__ src, T* __restrict__ dst) {
  const int b = blockIdx.x;
  if (b >= nb) return;
  const int k = ks[b];
  if (k <= 0) return;
  const RkLeafDesc s = src_desc[b], d = dst_desc[b];
  const int m = d.m, n = d.n, k0 = kcur[b];
  const T* A1 = src + s.ws_off;
  const T* B1 = A1 + (size_t)m * s.kcap;
  T* A2 = dst + d.ws_off;
  T* B2 = A2 + (size_t)m * d.kcap;
  for (int e = threadIdx.x; e < m * k; e += blockDim.x) A2[(size_t)k0 * m + e] = scale_by(A1[e], w);
  for (int e = threadIdx.x; e < n * k; e += blockDim.x) B2[(size_t)k0 * n + e] = B1[e];
}

// The leaves in `order` hold [A | A_s], [B | B_s] (kcur[b] + the stratum's columns = kcat[b]):
// their full block D = A B^T + A_s B_s^T (the two products summed separately, in increasing
// column order, then added: the order of eval() + axpy in formattedAddParts) goes through
// `scratch` (m x n at dof[item]) and comes back into the slot as the exact rank-min(m, n)
// factorisation D = D I^T (m >= n) or I D^T (m < n), whose truncation is the SVD of D.
template <typename T>
__global__ void __launch_bounds__(256) exact_kernel(const RkLeafDesc* __restrict__ leaves,
                                                    const int* __restrict__ order, int count,
                                                    const int* __restrict__ kcur, const int* __restrict__ kcat,
                                                    const long long* __restrict__ dof, T* ws, T* scratch) {
  typedef typename Traits<T>::wide W;
  const int item = blockIdx.x;
  if (item >= count) return;
  const int b = order[item];
  const RkLeafDesc d = leaves[b];
  const int m = d.m, n = d.n, k0 = kcur[b], k1 = kcat[b];
  T* A = ws + d.ws_off;
  T* B = A + (size_t)m * d.kcap;
  T* D = scratch + dof[item];
  for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
    const int i = e % m, j = e / m;
    W s0 = zero<W>(), s1 = zero<W>();
    for (int l = 0; l < k0; ++l) s0 = upd(widen(A[(size_t)l * m + i]), widen(B[(size_t)l * n + j]), s0);
    for (int l = k0; l < k1; ++l) s1 = upd(widen(A[(size_t)l * m + i]), widen(B[(size_t)l * n + j]), s1);
    D[e] = narrow<T>(s0 + s1);
  }
  __syncthreads();
  if (m >= n) {
    for (int e = threadIdx.x; e < m * n; e += blockDim.x) A[e] = D[e];  // A = D (m x n)
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) B[e] = (e % (n + 1) == 0) ? one<T>() : zero<T>();
  } else {
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] = (e % (m + 1) == 0) ? one<T>() : zero<T>();
    for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
      const int i = e % m, j = e / m;
      B[(size_t)i * n + j] = D[e];  // B = D^T (n x m)
    }
  }
}

}  // namespace

template <typename T>
void launch_scale_a(const RkLeafDesc* d_leaves, const int* d_order, int count, const int* ranks, double w, T* ws,
                    cudaStream_t s) {
  if (count <= 0) return;
  scale_a_kernel<T><<<count, 256, 0, s>>>(d_leaves, d_order, count, ranks, w, ws);
}

template <typename T>
void launch_append_factors(const RkLeafDesc* src_desc, const RkLeafDesc* dst_desc, int nb, const int* kcur,
                           const int* ks, double w, const T* src, T* dst, cudaStream_t s) {
  if (nb <= 0) return;
  append_kernel<T><<<nb, 256, 0, s>>>(src_desc, dst_desc, nb, kcur, ks, w, src, dst);
}

template <typename T>
void launch_exact_factors(const RkLeafDesc* d_leaves, const int* d_order, int count, const int* kcur,
                          const int* kcat, const long long* dof, T* ws, T* scratch, cudaStream_t s) {
  if (count <= 0) return;
  exact_kernel<T><<<count, 256, 0, s>>>(d_leaves, d_order, count, kcur, kcat, dof, ws, scratch);
}

#define HB_INST(T)                                                                                          \
  template void launch_scale_a<T>(const RkLeafDesc*, const int*, int, const int*, double, T*, cudaStream_t); \
  template void launch_append_factors<T>(const RkLeafDesc*, const RkLeafDesc*, int, const int*, const int*,  \
                                         double, const T*, T*, cudaStream_t);                                \
  template void launch_exact_factors<T>(const RkLeafDesc*, const int*, int, const int*, const int*,          \
                                        const long long*, T*, T*, cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
