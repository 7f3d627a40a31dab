// CTA-wide reductions used by the per-leaf kernels (ACA, truncation).  All of them are
// deterministic: the combination order depends only on the CTA shape.
#pragma once
#include <cfloat>

#include "common.cuh"

namespace hmatb200 {

struct KeyIdx {
  double key;
  int idx;
};

// "a before b" for the first-index-of-maximum rule of BLAS i?amax.
__device__ inline bool amax_better(const KeyIdx& b, const KeyIdx& a) {
  return b.idx >= 0 && (a.idx < 0 || b.key > a.key || (b.key == a.key && b.idx < a.idx));
}
// "b before a" for the first-index-of-strict-minimum rule of findMinRow/findMinCol.
__device__ inline bool amin_better(const KeyIdx& b, const KeyIdx& a) {
  return b.idx >= 0 && (a.idx < 0 || b.key < a.key || (b.key == a.key && b.idx < a.idx));
}

template <bool MAX>
__device__ inline KeyIdx warp_arg(KeyIdx v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    KeyIdx o;
    o.key = __shfl_down_sync(0xffffffffu, v.key, off);
    o.idx = __shfl_down_sync(0xffffffffu, v.idx, off);
    if (MAX ? amax_better(o, v) : amin_better(o, v)) v = o;
  }
  return v;
}

// Shared scratch for one CTA's reductions (up to 32 warps).
struct RedScratch {
  double d[32];
  double d2[32];
  int i[32];
  int flag;
  KeyIdx res;
  KeyIdx res2;
};

template <bool MAX>
__device__ inline KeyIdx block_arg(KeyIdx v, RedScratch& s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_arg<MAX>(v);
  __syncthreads();
  if (lane == 0) {
    s.d[warp] = v.key;
    s.i[warp] = v.idx;
  }
  __syncthreads();
  if (warp == 0) {
    KeyIdx w;
    w.key = lane < nw ? s.d[lane] : 0.0;
    w.idx = lane < nw ? s.i[lane] : -1;
    w = warp_arg<MAX>(w);
    if (lane == 0) s.res = w;
  }
  __syncthreads();
  return s.res;
}

// Two independent arg-max reductions in one pass.
__device__ inline void block_argmax2(KeyIdx& a, KeyIdx& b, RedScratch& s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a = warp_arg<true>(a);
  b = warp_arg<true>(b);
  __syncthreads();
  if (lane == 0) {
    s.d[warp] = a.key;
    s.i[warp] = a.idx;
    s.d2[warp] = b.key;
  }
  __syncthreads();
  if (warp == 0) {
    KeyIdx w;
    w.key = lane < nw ? s.d[lane] : 0.0;
    w.idx = lane < nw ? s.i[lane] : -1;
    w = warp_arg<true>(w);
    if (lane == 0) s.res = w;
  }
  __syncthreads();
  // second reduction reuses the index slots
  if (lane == 0) s.i[warp] = b.idx;
  __syncthreads();
  if (warp == 0) {
    KeyIdx w;
    w.key = lane < nw ? s.d2[lane] : 0.0;
    w.idx = lane < nw ? s.i[lane] : -1;
    w = warp_arg<true>(w);
    if (lane == 0) s.res2 = w;
  }
  __syncthreads();
  a = s.res;
  b = s.res2;
}

__device__ inline bool block_any(bool v, RedScratch& s) {
  __syncthreads();
  if (threadIdx.x == 0) s.flag = 0;
  __syncthreads();
  if (__any_sync(0xffffffffu, v) && (threadIdx.x & 31) == 0) atomicOr(&s.flag, 1);
  __syncthreads();
  return s.flag != 0;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;
}
__device__ inline cdouble warp_sum(cdouble v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, off);
    v.y += __shfl_down_sync(0xffffffffu, v.y, off);
  }
  return v;
}
// Broadcast lane 0's value to the whole warp.
__device__ inline double warp_bcast(double v) { return __shfl_sync(0xffffffffu, v, 0); }
__device__ inline cdouble warp_bcast(cdouble v) {
  return cdouble{__shfl_sync(0xffffffffu, v.x, 0), __shfl_sync(0xffffffffu, v.y, 0)};
}

__device__ inline double block_sum(double v, RedScratch& s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) s.d[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double w = lane < nw ? s.d[lane] : 0.0;
    w = warp_sum(w);
    if (lane == 0) s.d2[0] = w;
  }
  __syncthreads();
  return s.d2[0];
}

}  // namespace hmatb200
