// Scalar traits, kernel functions and small device helpers shared by the B200 engine's
// CUDA kernels (sm_100a).
//
// Scalar types mirror hmat-oss's four value types (data_types.hpp:76-82):
//   float (S), double (D), cfloat (C), cdouble (Z).
// Unlike the reference, whose S/C types compress in double and only store in single
// precision (compression.cpp:746-773, fromdouble.cpp:37-99), the S/C engines here run
// assembly, ACA and gemv in single precision and keep FP64 only for the stopping-norm
// estimate of ACA+ and for the QR/SVD of the truncation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hmatb200 {

struct cfloat {
  float x, y;
};
struct cdouble {
  double x, y;
};

__host__ __device__ inline cfloat mk(float a, float b) { return cfloat{a, b}; }
__host__ __device__ inline cdouble mk(double a, double b) { return cdouble{a, b}; }

#define HB_CPLX_OPS(C, R)                                                                         \
  __host__ __device__ inline C operator+(C a, C b) { return C{a.x + b.x, a.y + b.y}; }            \
  __host__ __device__ inline C operator-(C a, C b) { return C{a.x - b.x, a.y - b.y}; }            \
  __host__ __device__ inline C operator-(C a) { return C{-a.x, -a.y}; }                           \
  __host__ __device__ inline C operator*(C a, C b) { return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; } \
  __host__ __device__ inline C operator*(R s, C b) { return C{s * b.x, s * b.y}; }                \
  __host__ __device__ inline C operator*(C b, R s) { return C{s * b.x, s * b.y}; }                \
  __host__ __device__ inline bool operator==(C a, C b) { return a.x == b.x && a.y == b.y; }       \
  __host__ __device__ inline bool operator!=(C a, C b) { return !(a == b); }
HB_CPLX_OPS(cfloat, float)
HB_CPLX_OPS(cdouble, double)
#undef HB_CPLX_OPS

template <typename T>
struct Traits;

template <>
struct Traits<float> {
  typedef float real;
  typedef double wide;  // FP64 companion used for norms and the truncation
  static const bool is_complex = false;
  static const int code = 0;
};
template <>
struct Traits<double> {
  typedef double real;
  typedef double wide;
  static const bool is_complex = false;
  static const int code = 1;
};
template <>
struct Traits<cfloat> {
  typedef float real;
  typedef cdouble wide;
  static const bool is_complex = true;
  static const int code = 2;
};
template <>
struct Traits<cdouble> {
  typedef double real;
  typedef cdouble wide;
  static const bool is_complex = true;
  static const int code = 3;
};

// |x|^2 in double (squaredNorm, data_types.hpp:105-132)
__device__ __host__ inline double abs2(float a) { return (double)a * (double)a; }
__device__ __host__ inline double abs2(double a) { return a * a; }
__device__ __host__ inline double abs2(cfloat a) { return (double)a.x * a.x + (double)a.y * a.y; }
__device__ __host__ inline double abs2(cdouble a) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));  // no contraction: the host rounding
#else
  return a.x * a.x + a.y * a.y;
#endif
}

// Ranking key of BLAS i?amax: |x| for real, |Re|+|Im| for complex (blas_overloads.hpp:159-180).
__device__ inline double amax_key(float a) { return fabs((double)a); }
__device__ inline double amax_key(double a) { return fabs(a); }
__device__ inline double amax_key(cfloat a) { return fabs((double)a.x) + fabs((double)a.y); }
__device__ inline double amax_key(cdouble a) { return fabs(a.x) + fabs(a.y); }

__device__ __host__ inline float conjg(float a) { return a; }
__device__ __host__ inline double conjg(double a) { return a; }
__device__ __host__ inline cfloat conjg(cfloat a) { return cfloat{a.x, -a.y}; }
__device__ __host__ inline cdouble conjg(cdouble a) { return cdouble{a.x, -a.y}; }

__device__ __host__ inline double real_part(double a) { return a; }
__device__ __host__ inline double real_part(cdouble a) { return a.x; }

template <typename T>
__device__ __host__ inline T zero() {
  return T{};
}
template <>
__device__ __host__ inline float zero<float>() {
  return 0.f;
}
template <>
__device__ __host__ inline double zero<double>() {
  return 0.0;
}

template <typename T>
__device__ __host__ inline T one();
template <>
__device__ __host__ inline float one<float>() {
  return 1.f;
}
template <>
__device__ __host__ inline double one<double>() {
  return 1.0;
}
template <>
__device__ __host__ inline cfloat one<cfloat>() {
  return cfloat{1.f, 0.f};
}
template <>
__device__ __host__ inline cdouble one<cdouble>() {
  return cdouble{1.0, 0.0};
}

__device__ __host__ inline bool is_zero_val(float a) { return a == 0.f; }
__device__ __host__ inline bool is_zero_val(double a) { return a == 0.0; }
__device__ __host__ inline bool is_zero_val(cfloat a) { return a.x == 0.f && a.y == 0.f; }
__device__ __host__ inline bool is_zero_val(cdouble a) { return a.x == 0.0 && a.y == 0.0; }

// Widening / narrowing between the storage type and its FP64 companion.
__device__ __host__ inline double widen(float a) { return (double)a; }
__device__ __host__ inline double widen(double a) { return a; }
__device__ __host__ inline cdouble widen(cfloat a) { return cdouble{(double)a.x, (double)a.y}; }
__device__ __host__ inline cdouble widen(cdouble a) { return a; }
template <typename T>
__device__ __host__ inline T narrow(typename Traits<T>::wide a);
template <>
__device__ __host__ inline float narrow<float>(double a) {
  return (float)a;
}
template <>
__device__ __host__ inline double narrow<double>(double a) {
  return a;
}
template <>
__device__ __host__ inline cfloat narrow<cfloat>(cdouble a) {
  return cfloat{(float)a.x, (float)a.y};
}
template <>
__device__ __host__ inline cdouble narrow<cdouble>(cdouble a) {
  return a;
}

#ifdef __CUDACC__  // device arithmetic (host translation units only need the types above)
// acc + a * b with a single rounding per real multiply-add (the FMA form OpenBLAS axpy
// kernels use on x86).
__device__ inline float fmadd(float a, float b, float acc) { return fmaf(a, b, acc); }
__device__ inline double fmadd(double a, double b, double acc) { return fma(a, b, acc); }
__device__ inline cfloat fmadd(cfloat a, cfloat b, cfloat acc) {
  return cfloat{fmaf(-a.y, b.y, fmaf(a.x, b.x, acc.x)), fmaf(a.y, b.x, fmaf(a.x, b.y, acc.y))};
}
__device__ inline cdouble fmadd(cdouble a, cdouble b, cdouble acc) {
  return cdouble{fma(-a.y, b.y, fma(a.x, b.x, acc.x)), fma(a.y, b.x, fma(a.x, b.y, acc.y))};
}

// 1 / z for the pivot scaling: conj(z) / |z|^2, the textbook form the reference's
// -ffast-math build evaluates, each operation rounded separately in FP64.
__device__ inline float recip(float a) { return 1.0f / a; }
__device__ inline double recip(double a) { return __ddiv_rn(1.0, a); }
__device__ inline cfloat recip(cfloat a) {
  float d = a.x * a.x + a.y * a.y;
  return cfloat{a.x / d, -a.y / d};
}
__device__ inline cdouble recip(cdouble a) {
  double d = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
  return cdouble{__ddiv_rn(a.x, d), __ddiv_rn(-a.y, d)};
}

// Residual updates and scalings of ACA (v + a * x, v * s).  The FP64 engines round every
// product and sum separately, as the reference's CPU arithmetic does (an FMA would round
// once and change which of two tied pivot candidates wins); the FP32 engines use FMA.
__device__ inline float upd(float a, float x, float v) { return fmaf(a, x, v); }
__device__ inline cfloat upd(cfloat a, cfloat x, cfloat v) { return fmadd(a, x, v); }
__device__ inline double upd(double a, double x, double v) { return __dadd_rn(v, __dmul_rn(a, x)); }
__device__ inline cdouble upd(cdouble a, cdouble x, cdouble v) {
  const double re = __dsub_rn(__dmul_rn(a.x, x.x), __dmul_rn(a.y, x.y));
  const double im = __dadd_rn(__dmul_rn(a.x, x.y), __dmul_rn(a.y, x.x));
  return cdouble{__dadd_rn(v.x, re), __dadd_rn(v.y, im)};
}
__device__ inline float mul_rn(float v, float s) { return v * s; }
__device__ inline cfloat mul_rn(cfloat v, cfloat s) { return v * s; }
__device__ inline double mul_rn(double v, double s) { return __dmul_rn(v, s); }
__device__ inline cdouble mul_rn(cdouble v, cdouble s) {
  return cdouble{__dsub_rn(__dmul_rn(v.x, s.x), __dmul_rn(v.y, s.y)),
                 __dadd_rn(__dmul_rn(v.x, s.y), __dmul_rn(v.y, s.x))};
}
#endif  // __CUDACC__

// ------------------------------------------------------------------------------------
// Interaction kernels.  Entries are evaluated from cluster-ordered coordinates; the
// FP64 path follows the same IEEE operation order as the reference harness's callbacks
// (no contraction), so regularised-Laplace entries are bit-identical to the CPU ones.
// ------------------------------------------------------------------------------------

enum KernelKind { kLaplaceReg = 0, kExpCov = 1, kHelmholtzReg = 2 };

// Multi-strata kernels (the reference's advanced_compute callbacks with prepare's
// number_of_strata, hmat.h:552-583): the kernel is the sum of its strata, stratum q being w_q
// times the kernel with its parameter replaced by a_q (the correlation length of the
// exponential covariance, with no nugget; the regularisation of the Laplace kernel; the
// wavenumber of the Helmholtz kernel, whose amplitude keeps delta).  `strata` is a device array
// a_0 .. a_{nstrata-1}, w_0 .. w_{nstrata-1}; eval_sum() evaluates the sum in stratum order.
// The ACA of one stratum q runs eval() on the plain kernel with the parameter a_q and nugget 0;
// w_q multiplies its A factor afterwards.
constexpr int kMaxStrata = 8;
struct KernelParams {
  int kind;
  double delta;       // r + delta regularisation
  double ell;         // correlation length
  double nugget;      // diagonal term of the covariance
  double wavenumber;  // Helmholtz k
  int nstrata = 0;    // 0: a plain kernel
  const double* strata = nullptr;
};

// Cluster-ordered coordinates of the row and column points (the same arrays when the
// matrix is built on one tree) and their client numbers (for the covariance nugget).
struct Points {
  const double *rx, *ry, *rz;
  const double *cx, *cy, *cz;
  const int* rid;
  const int* cid;
  // Optional per-row-point kernel parameter (cluster order), replacing the kernel's own ell
  // (exponential covariance), delta (regularised Laplace and Helmholtz amplitude) or
  // wavenumber (Helmholtz phase) -- see param_of.
  const double* rprm = nullptr;
};

#define HB_FOUR_PI 12.566370614359172  // 4 * M_PI in double

#ifdef __CUDACC__  // device arithmetic continues

__device__ inline double dist_fp64(const Points& p, int i, int j) {
  double dx = __dsub_rn(p.rx[i], p.cx[j]);
  double dy = __dsub_rn(p.ry[i], p.cy[j]);
  double dz = __dsub_rn(p.rz[i], p.cz[j]);
  double s = __dmul_rn(dx, dx);
  s = __dadd_rn(s, __dmul_rn(dy, dy));
  s = __dadd_rn(s, __dmul_rn(dz, dz));
  return __dsqrt_rn(s);
}

// Single-precision distance: the coordinate differences are taken in FP64 (so close
// points keep their relative accuracy) and the rest runs in FP32.
__device__ inline float dist_fp32(const Points& p, int i, int j) {
  float dx = (float)(p.rx[i] - p.cx[j]);
  float dy = (float)(p.ry[i] - p.cy[j]);
  float dz = (float)(p.rz[i] - p.cz[j]);
  return sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
}

template <typename T>
struct KernelEval;

// The kernel's parameter for row point i: its own (per-point array) or the kernel's.
__device__ inline double param_of(const Points& p, int i, double own) { return p.rprm ? p.rprm[i] : own; }

template <>
struct KernelEval<double> {
  __device__ static inline double eval(const KernelParams& k, const Points& p, int i, int j) {
    double r = dist_fp64(p, i, j);
    if (k.kind == kLaplaceReg) return __ddiv_rn(1.0, __dmul_rn(HB_FOUR_PI, __dadd_rn(r, param_of(p, i, k.delta))));
    double v = exp(__ddiv_rn(-r, param_of(p, i, k.ell)));
    if (p.rid[i] == p.cid[j]) v = __dadd_rn(v, k.nugget);
    return v;
  }
  // The strata summed in order: w (1 / (4 pi (r + a))) or w exp(-r / a), FP64 operations in
  // the order of the reference's strata callbacks.
  __device__ static inline double eval_sum(const KernelParams& k, const Points& p, int i, int j) {
    const double r = dist_fp64(p, i, j);
    double sum = 0.0;
    for (int q = 0; q < k.nstrata; ++q) {
      const double a = k.strata[q], w = k.strata[k.nstrata + q];
      const double v = k.kind == kLaplaceReg ? __ddiv_rn(1.0, __dmul_rn(HB_FOUR_PI, __dadd_rn(r, a)))
                                             : exp(__ddiv_rn(-r, a));
      sum = __dadd_rn(sum, __dmul_rn(w, v));
    }
    return sum;
  }
};

template <>
struct KernelEval<float> {
  __device__ static inline float eval(const KernelParams& k, const Points& p, int i, int j) {
    float r = dist_fp32(p, i, j);
    if (k.kind == kLaplaceReg) return 1.0f / ((float)HB_FOUR_PI * (r + (float)param_of(p, i, k.delta)));
    float v = expf(-r / (float)param_of(p, i, k.ell));
    if (p.rid[i] == p.cid[j]) v += (float)k.nugget;
    return v;
  }
  __device__ static inline float eval_sum(const KernelParams& k, const Points& p, int i, int j) {
    const float r = dist_fp32(p, i, j);
    float sum = 0.0f;
    for (int q = 0; q < k.nstrata; ++q) {
      const float a = (float)k.strata[q], w = (float)k.strata[k.nstrata + q];
      sum += w * (k.kind == kLaplaceReg ? 1.0f / ((float)HB_FOUR_PI * (r + a)) : expf(-r / a));
    }
    return sum;
  }
};

template <>
struct KernelEval<cdouble> {
  __device__ static inline cdouble eval(const KernelParams& k, const Points& p, int i, int j) {
    double r = dist_fp64(p, i, j);
    double s = __ddiv_rn(1.0, __dmul_rn(HB_FOUR_PI, __dadd_rn(r, k.delta)));
    double sn, cs;
    sincos(__dmul_rn(param_of(p, i, k.wavenumber), r), &sn, &cs);
    return cdouble{cs * s, sn * s};
  }
  // w (cos(a r) s), w (sin(a r) s), real and imaginary parts summed in stratum order.
  __device__ static inline cdouble eval_sum(const KernelParams& k, const Points& p, int i, int j) {
    const double r = dist_fp64(p, i, j);
    const double s = __ddiv_rn(1.0, __dmul_rn(HB_FOUR_PI, __dadd_rn(r, k.delta)));
    double re = 0.0, im = 0.0;
    for (int q = 0; q < k.nstrata; ++q) {
      const double w = k.strata[k.nstrata + q];
      double sn, cs;
      sincos(__dmul_rn(k.strata[q], r), &sn, &cs);
      re = __dadd_rn(re, __dmul_rn(w, __dmul_rn(cs, s)));
      im = __dadd_rn(im, __dmul_rn(w, __dmul_rn(sn, s)));
    }
    return cdouble{re, im};
  }
};

template <>
struct KernelEval<cfloat> {
  __device__ static inline cfloat eval(const KernelParams& k, const Points& p, int i, int j) {
    // The phase k*r is formed in FP64: at 10 points per wavelength k*r reaches
    // hundreds of radians, where an FP32 argument would lose most of its digits.
    double r = dist_fp64(p, i, j);
    float s = 1.0f / ((float)HB_FOUR_PI * ((float)r + (float)k.delta));
    double kr = param_of(p, i, k.wavenumber) * r;
    float ph = (float)(kr - 6.283185307179586 * rint(kr * 0.15915494309189535));
    float sn, cs;
    sincosf(ph, &sn, &cs);
    return cfloat{cs * s, sn * s};
  }
  __device__ static inline cfloat eval_sum(const KernelParams& k, const Points& p, int i, int j) {
    const double r = dist_fp64(p, i, j);
    const float s = 1.0f / ((float)HB_FOUR_PI * ((float)r + (float)k.delta));
    float re = 0.0f, im = 0.0f;
    for (int q = 0; q < k.nstrata; ++q) {
      const float w = (float)k.strata[k.nstrata + q];
      const double kr = k.strata[q] * r;
      float sn, cs;
      sincosf((float)(kr - 6.283185307179586 * rint(kr * 0.15915494309189535)), &sn, &cs);
      re += w * (cs * s);
      im += w * (sn * s);
    }
    return cfloat{re, im};
  }
};

#endif  // __CUDACC__

// ------------------------------------------------------------------------------------
// Leaf error codes, written per leaf by the device phases and mapped to a non-zero C
// return code on the host.
// ------------------------------------------------------------------------------------
enum LeafStatus {
  kLeafOk = 0,
  kLeafAcaCapacity = 1,   // ACA reached its rank capacity before converging
  kLeafSvdNoConverge = 2, // Jacobi sweeps hit their cap (result still used, flagged)
  kLeafBadShape = 3,
};

}  // namespace hmatb200
