/* Prototype-only CBLAS header (public CBLAS interface, LP64 ints) used to compile
 * the reference library for the oracle build.  Complex arguments are passed as
 * untyped pointers, which is how the CBLAS standard defines them.  The symbols
 * are resolved against the OpenBLAS shipped in the image.  Test infrastructure
 * only: nothing in the product links this header. */
#ifndef ORACLE_REFSHIM_CBLAS_H
#define ORACLE_REFSHIM_CBLAS_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
typedef enum CBLAS_ORDER CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO CBLAS_UPLO;
typedef enum CBLAS_DIAG CBLAS_DIAG;
typedef enum CBLAS_SIDE CBLAS_SIDE;

void cblas_saxpy(int n, float a, const float* x, int incx, float* y, int incy);
void cblas_daxpy(int n, double a, const double* x, int incx, double* y, int incy);
void cblas_caxpy(int n, const void* a, const void* x, int incx, void* y, int incy);
void cblas_zaxpy(int n, const void* a, const void* x, int incx, void* y, int incy);

float cblas_sdot(int n, const float* x, int incx, const float* y, int incy);
double cblas_ddot(int n, const double* x, int incx, const double* y, int incy);
void cblas_cdotu_sub(int n, const void* x, int incx, const void* y, int incy, void* ret);
void cblas_zdotu_sub(int n, const void* x, int incx, const void* y, int incy, void* ret);
void cblas_cdotc_sub(int n, const void* x, int incx, const void* y, int incy, void* ret);
void cblas_zdotc_sub(int n, const void* x, int incx, const void* y, int incy, void* ret);

size_t cblas_isamax(int n, const float* x, int incx);
size_t cblas_idamax(int n, const double* x, int incx);
size_t cblas_icamax(int n, const void* x, int incx);
size_t cblas_izamax(int n, const void* x, int incx);

void cblas_sscal(int n, float a, float* x, int incx);
void cblas_dscal(int n, double a, double* x, int incx);
void cblas_cscal(int n, const void* a, void* x, int incx);
void cblas_zscal(int n, const void* a, void* x, int incx);

void cblas_sgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, int m, int n, float alpha, const float* a, int lda,
                 const float* x, int incx, float beta, float* y, int incy);
void cblas_dgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, int m, int n, double alpha, const double* a, int lda,
                 const double* x, int incx, double beta, double* y, int incy);
void cblas_cgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, int m, int n, const void* alpha, const void* a, int lda,
                 const void* x, int incx, const void* beta, void* y, int incy);
void cblas_zgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, int m, int n, const void* alpha, const void* a, int lda,
                 const void* x, int incx, const void* beta, void* y, int incy);

void cblas_sger(CBLAS_ORDER o, int m, int n, float alpha, const float* x, int incx, const float* y, int incy,
                float* a, int lda);
void cblas_dger(CBLAS_ORDER o, int m, int n, double alpha, const double* x, int incx, const double* y, int incy,
                double* a, int lda);
void cblas_cgeru(CBLAS_ORDER o, int m, int n, const void* alpha, const void* x, int incx, const void* y,
                 int incy, void* a, int lda);
void cblas_zgeru(CBLAS_ORDER o, int m, int n, const void* alpha, const void* x, int incx, const void* y,
                 int incy, void* a, int lda);

void cblas_sgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k, float alpha,
                 const float* a, int lda, const float* b, int ldb, float beta, float* c, int ldc);
void cblas_dgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double* a, int lda, const double* b, int ldb, double beta, double* c, int ldc);
void cblas_cgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k, const void* alpha,
                 const void* a, int lda, const void* b, int ldb, const void* beta, void* c, int ldc);
void cblas_zgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k, const void* alpha,
                 const void* a, int lda, const void* b, int ldb, const void* beta, void* c, int ldc);

void cblas_strmm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 float alpha, const float* a, int lda, float* b, int ldb);
void cblas_dtrmm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 double alpha, const double* a, int lda, double* b, int ldb);
void cblas_ctrmm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 const void* alpha, const void* a, int lda, void* b, int ldb);
void cblas_ztrmm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 const void* alpha, const void* a, int lda, void* b, int ldb);
void cblas_strsm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 float alpha, const float* a, int lda, float* b, int ldb);
void cblas_dtrsm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 double alpha, const double* a, int lda, double* b, int ldb);
void cblas_ctrsm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 const void* alpha, const void* a, int lda, void* b, int ldb);
void cblas_ztrsm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, int m, int n,
                 const void* alpha, const void* a, int lda, void* b, int ldb);
#ifdef __cplusplus
}
#endif
#endif
