/*
 * Declaration-only stand-in for the two LAPACK routines the digHolo
 * reference calls through <mkl_lapack.h> (digHolo.cpp:63, used at
 * digHolo.cpp:3043 cgesvd and digHolo.cpp:3224 sgels).  The definitions in
 * lapack_shim.cpp forward to the Fortran-ABI OpenBLAS symbols cgesvd_ and
 * sgels_.  TEST INFRASTRUCTURE ONLY (oracle build); not linked by the product.
 */
#ifndef DIGHOLO_ORACLE_MKL_LAPACK_SHIM_H
#define DIGHOLO_ORACLE_MKL_LAPACK_SHIM_H

typedef struct { float real; float imag; } MKL_Complex8;
typedef int MKL_INT;

#ifdef __cplusplus
extern "C" {
#endif

void cgesvd(const char* jobu, const char* jobvt, const MKL_INT* m, const MKL_INT* n,
            MKL_Complex8* a, const MKL_INT* lda, float* s, MKL_Complex8* u, const MKL_INT* ldu,
            MKL_Complex8* vt, const MKL_INT* ldvt, MKL_Complex8* work, const MKL_INT* lwork,
            float* rwork, MKL_INT* info);

void sgels(const char* trans, const MKL_INT* m, const MKL_INT* n, const MKL_INT* nrhs,
           float* a, const MKL_INT* lda, float* b, const MKL_INT* ldb,
           float* work, const MKL_INT* lwork, MKL_INT* info);

#ifdef __cplusplus
}
#endif

#endif
