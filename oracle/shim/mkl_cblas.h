/*
 * Declaration-only stand-in for the two CBLAS routines the digHolo reference
 * calls through <mkl_cblas.h> (digHolo.cpp:65; cblas_cgemm at
 * digHolo.cpp:3090, cblas_cgemv at digHolo.cpp:5029 and 9597).  The enum
 * values are the standard CBLAS ones, so the calls bind directly to the
 * OpenBLAS exports of the same names.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef DIGHOLO_ORACLE_MKL_CBLAS_SHIM_H
#define DIGHOLO_ORACLE_MKL_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_cgemm(const enum CBLAS_LAYOUT layout, const enum CBLAS_TRANSPOSE transa,
                 const enum CBLAS_TRANSPOSE transb, const int m, const int n, const int k,
                 const void* alpha, const void* a, const int lda, const void* b, const int ldb,
                 const void* beta, void* c, const int ldc);

void cblas_cgemv(const enum CBLAS_LAYOUT layout, const enum CBLAS_TRANSPOSE trans,
                 const int m, const int n, const void* alpha, const void* a, const int lda,
                 const void* x, const int incx, const void* beta, void* y, const int incy);

#ifdef __cplusplus
}
#endif

#endif
