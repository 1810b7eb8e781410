/*
 * Forwarders from the MKL-style LAPACK names the digHolo reference calls
 * (cgesvd, sgels; digHolo.cpp:3043, 3224) to the Fortran-ABI OpenBLAS
 * exports (cgesvd_, sgels_).  Each CHARACTER*1 argument gets its hidden
 * length argument (1) appended, as gfortran-built LAPACK expects.
 * TEST INFRASTRUCTURE ONLY: part of the oracle build in oracle/_ref.
 */
#include <cstddef>
#include "mkl_lapack.h"

extern "C" {
void cgesvd_(const char* jobu, const char* jobvt, const int* m, const int* n, MKL_Complex8* a,
             const int* lda, float* s, MKL_Complex8* u, const int* ldu, MKL_Complex8* vt,
             const int* ldvt, MKL_Complex8* work, const int* lwork, float* rwork, int* info,
             size_t len_jobu, size_t len_jobvt);
void sgels_(const char* trans, const int* m, const int* n, const int* nrhs, float* a,
            const int* lda, float* b, const int* ldb, float* work, const int* lwork, int* info,
            size_t len_trans);

void cgesvd(const char* jobu, const char* jobvt, const MKL_INT* m, const MKL_INT* n,
            MKL_Complex8* a, const MKL_INT* lda, float* s, MKL_Complex8* u, const MKL_INT* ldu,
            MKL_Complex8* vt, const MKL_INT* ldvt, MKL_Complex8* work, const MKL_INT* lwork,
            float* rwork, MKL_INT* info)
{
    cgesvd_(jobu, jobvt, m, n, a, lda, s, u, ldu, vt, ldvt, work, lwork, rwork, info, 1, 1);
}

void sgels(const char* trans, const MKL_INT* m, const MKL_INT* n, const MKL_INT* nrhs,
           float* a, const MKL_INT* lda, float* b, const MKL_INT* ldb,
           float* work, const MKL_INT* lwork, MKL_INT* info)
{
    sgels_(trans, m, n, nrhs, a, lda, b, ldb, work, lwork, info, 1);
}
}
