/* Prototype-only LAPACKE header (public LAPACKE interface, LP64) used to compile
 * the reference library for the oracle build.  The includer defines
 * lapack_complex_float / lapack_complex_double before including it.  Test
 * infrastructure only. */
#ifndef ORACLE_REFSHIM_LAPACKE_H
#define ORACLE_REFSHIM_LAPACKE_H
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;
#ifndef lapack_complex_float
#define lapack_complex_float float _Complex
#endif
#ifndef lapack_complex_double
#define lapack_complex_double double _Complex
#endif
#ifdef __cplusplus
extern "C" {
#endif
#define ORACLE_LAPACKE_DECL(P, T, R)                                                                  \
  lapack_int LAPACKE_##P##getrf(int l, lapack_int m, lapack_int n, T* a, lapack_int lda, lapack_int* ipiv); \
  lapack_int LAPACKE_##P##getri(int l, lapack_int n, T* a, lapack_int lda, const lapack_int* ipiv);      \
  lapack_int LAPACKE_##P##getrs(int l, char t, lapack_int n, lapack_int nrhs, const T* a, lapack_int lda, \
                                const lapack_int* ipiv, T* b, lapack_int ldb);                           \
  lapack_int LAPACKE_##P##geqrf(int l, lapack_int m, lapack_int n, T* a, lapack_int lda, T* tau);        \
  lapack_int LAPACKE_##P##gesdd(int l, char jobz, lapack_int m, lapack_int n, T* a, lapack_int lda, R* s,\
                                T* u, lapack_int ldu, T* vt, lapack_int ldvt);                           \
  lapack_int LAPACKE_##P##gesvd(int l, char ju, char jvt, lapack_int m, lapack_int n, T* a,              \
                                lapack_int lda, R* s, T* u, lapack_int ldu, T* vt, lapack_int ldvt,     \
                                R* superb);                                                              \
  lapack_int LAPACKE_##P##laswp(int l, lapack_int n, T* a, lapack_int lda, lapack_int k1, lapack_int k2, \
                                const lapack_int* ipiv, lapack_int incx);                                \
  lapack_int LAPACKE_##P##potrf(int l, char uplo, lapack_int n, T* a, lapack_int lda);
ORACLE_LAPACKE_DECL(s, float, float)
ORACLE_LAPACKE_DECL(d, double, double)
ORACLE_LAPACKE_DECL(c, lapack_complex_float, float)
ORACLE_LAPACKE_DECL(z, lapack_complex_double, double)
#undef ORACLE_LAPACKE_DECL
lapack_int LAPACKE_sormqr(int l, char side, char trans, lapack_int m, lapack_int n, lapack_int k,
                          const float* a, lapack_int lda, const float* tau, float* c, lapack_int ldc);
lapack_int LAPACKE_dormqr(int l, char side, char trans, lapack_int m, lapack_int n, lapack_int k,
                          const double* a, lapack_int lda, const double* tau, double* c, lapack_int ldc);
lapack_int LAPACKE_cunmqr(int l, char side, char trans, lapack_int m, lapack_int n, lapack_int k,
                          const lapack_complex_float* a, lapack_int lda, const lapack_complex_float* tau,
                          lapack_complex_float* c, lapack_int ldc);
lapack_int LAPACKE_zunmqr(int l, char side, char trans, lapack_int m, lapack_int n, lapack_int k,
                          const lapack_complex_double* a, lapack_int lda, const lapack_complex_double* tau,
                          lapack_complex_double* c, lapack_int ldc);
lapack_int LAPACKE_clacgv(lapack_int n, lapack_complex_float* x, lapack_int incx);
lapack_int LAPACKE_zlacgv(lapack_int n, lapack_complex_double* x, lapack_int incx);
#ifdef __cplusplus
}
#endif
#endif
