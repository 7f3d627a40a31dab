// Dense assembly of the non-admissible (full) leaves: every entry of every full leaf is
// one kernel evaluation, written once, column-major, into the full-leaf arena.  Restates
// the full branch of AssemblyFunction::assemble / SimpleFunction::assemble
// (assembly.cpp:66-91) with the interaction evaluated on the device.
#include "kernels.h"

namespace hmatb200 {
namespace {

// Each leaf is stored as row panels (one per output block of its rows), each panel
// column-major len x n.
template <typename T>
__global__ void __launch_bounds__(256) assemble_full_kernel(const FullLeafDesc* __restrict__ leaves, int nleaves,
                                                            const PanelDesc* __restrict__ panels, KernelParams kp,
                                                            Points pts, T* __restrict__ arena) {
  for (int leaf = blockIdx.x; leaf < nleaves; leaf += gridDim.x) {
    const FullLeafDesc d = leaves[leaf];
    for (int p = 0; p < d.npanel; ++p) {
      const PanelDesc P = panels[d.panel_first + p];
      T* F = arena + P.off;
      const int mn = P.len * d.n;
      for (int e = threadIdx.x; e < mn; e += blockDim.x) {
        const int i = e % P.len, j = e / P.len;
        // a multi-strata kernel's full leaves hold the sum of its strata
        F[e] = kp.nstrata > 0 ? KernelEval<T>::eval_sum(kp, pts, d.row_off + P.rs + i, d.col_off + j)
                              : KernelEval<T>::eval(kp, pts, d.row_off + P.rs + i, d.col_off + j);
      }
    }
  }
}

}  // namespace

template <typename T>
void launch_assemble_full(const FullLeafDesc* d_leaves, int nleaves, const PanelDesc* panels, const KernelParams& kp,
                          Points pts, T* arena, cudaStream_t s) {
  if (nleaves <= 0) return;
  int grid = persistent_grid(8);
  if (grid > nleaves) grid = nleaves;
  assemble_full_kernel<T><<<grid, 256, 0, s>>>(d_leaves, nleaves, panels, kp, pts, arena);
}

// Full leaves from their canonical payloads (m x n column-major at goff[leaf] in src) into
// the arena's row panels, for loading a stored matrix.
template <typename T>
__global__ void full_from_canonical_kernel(const FullLeafDesc* __restrict__ leaves, const long long* __restrict__ goff,
                                           int nleaves, const PanelDesc* __restrict__ panels,
                                           const T* __restrict__ src, T* __restrict__ arena) {
  for (int leaf = blockIdx.x; leaf < nleaves; leaf += gridDim.x) {
    const FullLeafDesc d = leaves[leaf];
    const T* F = src + goff[leaf];
    for (int p = 0; p < d.npanel; ++p) {
      const PanelDesc P = panels[d.panel_first + p];
      T* dst = arena + P.off;
      for (int e = threadIdx.x; e < P.len * d.n; e += blockDim.x) {
        const int i = e % P.len, j = e / P.len;
        dst[e] = F[(size_t)(P.rs + i) + (size_t)d.m * j];
      }
    }
  }
}

template <typename T>
void launch_full_from_canonical(const FullLeafDesc* d_leaves, const long long* goff, int nleaves,
                                const PanelDesc* panels, const T* src, T* arena, cudaStream_t s) {
  if (nleaves <= 0) return;
  int grid = persistent_grid(8);
  if (grid > nleaves) grid = nleaves;
  full_from_canonical_kernel<T><<<grid, 256, 0, s>>>(d_leaves, goff, nleaves, panels, src, arena);
}

// Segmented copy between two device buffers (relayout of stored leaves): segment g copies a
// rows x cols column-major block (fewer than 2^31 elements).  A CTA per segment, threads over
// elements: contiguous runs (cols = 1, or both leading dimensions equal to rows) as one flat
// copy, other blocks with 32-bit index arithmetic.
template <typename T>
__global__ void __launch_bounds__(256) copy_segments_kernel(const CopySeg* __restrict__ segs, int nseg,
                                                            const T* __restrict__ src, T* __restrict__ dst) {
  for (int g = blockIdx.x; g < nseg; g += gridDim.x) {
    const CopySeg c = segs[g];
    const T* s = src + c.src;
    T* d = dst + c.dst;
    const int count = c.rows * c.cols;
    if (c.cols == 1 || (c.src_ld == c.rows && c.dst_ld == c.rows)) {
      for (int e = threadIdx.x; e < count; e += blockDim.x) d[e] = s[e];
    } else {
      for (int e = threadIdx.x; e < count; e += blockDim.x) {
        const int q = e / c.rows, r = e - q * c.rows;
        d[r + (long long)q * c.dst_ld] = s[r + (long long)q * c.src_ld];
      }
    }
  }
}

template <typename T>
void launch_copy_segments(const CopySeg* segs, int nseg, const T* src, T* dst, cudaStream_t s) {
  if (nseg <= 0) return;
  int grid = persistent_grid(8);
  if (grid > nseg) grid = nseg;
  copy_segments_kernel<T><<<grid, 256, 0, s>>>(segs, nseg, src, dst);
}

template <typename T>
void preload_full_kernels() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, assemble_full_kernel<T>);
  cudaFuncGetAttributes(&a, full_from_canonical_kernel<T>);
  cudaFuncGetAttributes(&a, copy_segments_kernel<T>);
}

#define HB_INST(T)                                                                                      \
  template void preload_full_kernels<T>();                                                              \
  template void launch_assemble_full<T>(const FullLeafDesc*, int, const PanelDesc*, const KernelParams&, \
                                        Points, T*, cudaStream_t);                                       \
  template void launch_full_from_canonical<T>(const FullLeafDesc*, const long long*, int, const PanelDesc*, \
                                              const T*, T*, cudaStream_t);                                 \
  template void launch_copy_segments<T>(const CopySeg*, int, const T*, T*, cudaStream_t);
HB_INST(float)
HB_INST(double)
HB_INST(cfloat)
HB_INST(cdouble)
#undef HB_INST

}  // namespace hmatb200
