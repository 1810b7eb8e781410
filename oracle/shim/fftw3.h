/*
 * Declaration-only stand-in for the FFTW3 single-precision API, written for
 * this project so that the digHolo reference (digHolo.cpp, which includes
 * <fftw3.h> at digHolo.cpp:46) compiles on a machine without FFTW.
 *
 * TEST INFRASTRUCTURE ONLY: this header and fft_shim.cpp serve the oracle
 * build under oracle/_ref; nothing in the digholo_b200 product links them.
 *
 * Only the entry points the reference calls are declared (digHolo.cpp:6689,
 * 7172-7176, 7245-7249, 7416-7417, 7429-7434, 7483, 7502, 7516, 7579, 8734,
 * 11609, 11653, 13470, 15799, 15836, 16556-16559).  Semantics follow the
 * published FFTW3 manual: unnormalised transforms, FFTW_FORWARD = -1
 * exponent sign, the advanced "many" interface with inembed/onembed strides,
 * and the REDFT10 / REDFT01 real-even transforms (DCT-II / DCT-III).
 */
#ifndef DIGHOLO_ORACLE_FFTW3_SHIM_H
#define DIGHOLO_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s* fftwf_plan;
typedef int fftwf_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

/* r2r kinds, numbered as in the FFTW3 manual's enumeration order */
#define FFTW_R2HC 0
#define FFTW_HC2R 1
#define FFTW_DHT 2
#define FFTW_REDFT00 3
#define FFTW_REDFT01 4
#define FFTW_REDFT10 5
#define FFTW_REDFT11 6
#define FFTW_RODFT00 7
#define FFTW_RODFT01 8
#define FFTW_RODFT10 9
#define FFTW_RODFT11 10

extern const char fftwf_version[];

int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);

fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany,
                               fftwf_complex* in, const int* inembed, int istride, int idist,
                               fftwf_complex* out, const int* onembed, int ostride, int odist,
                               int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                   float* in, const int* inembed, int istride, int idist,
                                   fftwf_complex* out, const int* onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                   fftwf_complex* in, const int* inembed, int istride, int idist,
                                   float* out, const int* onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_r2r_2d(int n0, int n1, float* in, float* out,
                             fftwf_r2r_kind kind0, fftwf_r2r_kind kind1, unsigned flags);

void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_execute_r2r(const fftwf_plan p, float* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);

int fftwf_import_wisdom_from_filename(const char* filename);
int fftwf_export_wisdom_to_filename(const char* filename);
void fftwf_forget_wisdom(void);

#ifdef __cplusplus
}
#endif

#endif
