/*
 * A small FFT library exposing the subset of the FFTW3 single-precision API
 * that the digHolo reference calls (see fftw3.h for the call sites).  Written
 * for this project; it is NOT FFTW.
 *
 * TEST INFRASTRUCTURE ONLY.  It exists so that the unmodified reference
 * (digHolo.cpp) can be compiled and run here as the oracle / CPU baseline
 * (oracle/_ref/libdigholo_ref.so).  The digholo_b200 product never links it.
 *
 * Method (published, textbook):
 *   - complex transforms: recursive mixed-radix decimation-in-time
 *     Cooley-Tukey over the factorisation of n into 4, 2, 3, 5 and any
 *     remaining prime (done as a direct DFT of that radix);
 *   - real-to-complex of even length n: one complex FFT of length n/2 on the
 *     even/odd packed samples, then the standard split post-processing;
 *   - REDFT10 / REDFT01 (DCT-II / DCT-III as defined in the FFTW3 manual,
 *     unnormalised): direct O(n^2) sums with cached cosine tables.
 * All arithmetic is carried out in double precision and rounded to float on
 * output, so this library is more accurate than a float FFT; the oracle's
 * FFT stage therefore differs from FFTW only by float rounding.
 *
 * Plans are immutable after creation, and execution allocates its scratch
 * per call, so one plan may be executed concurrently from several threads
 * (the reference's thread pool does exactly that, digHolo.cpp:7184-7260).
 */
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

typedef std::complex<double> cd;

extern "C" const char fftwf_version[] = "digholo-oracle-fft-shim-1.0 (not FFTW)";

namespace {

const double kPi = 3.14159265358979323846264338327950288;

/* One length-n complex transform: factorisation plus a full twiddle table. */
struct Fft1d {
    int n = 0;
    int sign = -1;
    std::vector<int> factors;
    std::vector<cd> tw; /* tw[k] = exp(sign*2*pi*i*k/n), k < n */

    Fft1d(int n_, int sign_) : n(n_), sign(sign_) {
        int m = n;
        while (m % 4 == 0) { factors.push_back(4); m /= 4; }
        while (m % 2 == 0) { factors.push_back(2); m /= 2; }
        for (int p = 3; p * p <= m; p += 2) {
            while (m % p == 0) { factors.push_back(p); m /= p; }
        }
        if (m > 1) factors.push_back(m);
        if (factors.empty()) factors.push_back(1);
        tw.resize(n > 0 ? n : 1);
        for (int k = 0; k < n; k++) {
            const double a = sign * 2.0 * kPi * (double)k / (double)n;
            tw[k] = cd(std::cos(a), std::sin(a));
        }
    }

    /* out[0..len) = DFT of in[0], in[s], in[2s], ... (len = n / prod of used factors) */
    void rec(const cd* in, size_t s, cd* out, int len, int fi, cd* scratch) const {
        const int p = factors[fi];
        const int m = len / p;
        if (m == 1) {
            for (int j = 0; j < p; j++) out[j] = in[j * s];
        } else {
            for (int j = 0; j < p; j++) rec(in + j * s, s * p, out + j * m, m, fi + 1, scratch);
        }
        const int twStride = n / len; /* twiddle step for length len */
        if (p == 2) {
            for (int k = 0; k < m; k++) {
                const cd a = out[k];
                const cd b = out[k + m] * tw[(size_t)k * twStride];
                out[k] = a + b;
                out[k + m] = a - b;
            }
        } else if (p == 4) {
            const cd jrot = cd(0, (double)sign); /* exp(sign*i*pi/2) */
            for (int k = 0; k < m; k++) {
                const cd a0 = out[k];
                const cd a1 = out[k + m] * tw[(size_t)k * twStride];
                const cd a2 = out[k + 2 * m] * tw[(size_t)2 * k * twStride];
                const cd a3 = out[k + 3 * m] * tw[(size_t)3 * k * twStride];
                const cd s02 = a0 + a2, d02 = a0 - a2;
                const cd s13 = a1 + a3, d13 = (a1 - a3) * jrot;
                out[k] = s02 + s13;
                out[k + m] = d02 + d13;
                out[k + 2 * m] = s02 - s13;
                out[k + 3 * m] = d02 - d13;
            }
        } else {
            /* generic radix p: direct DFT of the p twiddled inputs */
            const int pStride = n / p;
            for (int k = 0; k < m; k++) {
                for (int q = 0; q < p; q++) {
                    scratch[q] = out[k + q * m] * tw[((size_t)q * k * twStride) % n];
                }
                for (int q2 = 0; q2 < p; q2++) {
                    cd acc = 0;
                    for (int q = 0; q < p; q++) acc += scratch[q] * tw[((size_t)q * q2 * pStride) % n];
                    out[k + q2 * m] = acc;
                }
            }
        }
    }

    void run(const cd* in, size_t s, cd* out) const {
        if (n == 1) { out[0] = in[0]; return; }
        int maxp = 1;
        for (int f : factors) maxp = f > maxp ? f : maxp;
        std::vector<cd> scratch(maxp);
        rec(in, s, out, n, 0, scratch.data());
    }
};

/* Real-input forward transform of even length n via a length n/2 complex FFT. */
struct Rfft1d {
    int n;
    Fft1d half;
    std::vector<cd> w; /* exp(-2 pi i k / n), k <= n/2 */
    explicit Rfft1d(int n_) : n(n_), half(n_ / 2, -1) {
        w.resize(n / 2 + 1);
        for (int k = 0; k <= n / 2; k++) {
            const double a = -2.0 * kPi * (double)k / (double)n;
            w[k] = cd(std::cos(a), std::sin(a));
        }
    }
    /* x: n real samples (double), X: n/2+1 outputs */
    void run(const double* x, cd* X) const {
        const int h = n / 2;
        std::vector<cd> z(h), Z(h);
        for (int j = 0; j < h; j++) z[j] = cd(x[2 * j], x[2 * j + 1]);
        half.run(z.data(), 1, Z.data());
        for (int k = 0; k <= h; k++) {
            const cd zk = Z[k % h];
            const cd zc = std::conj(Z[(h - k) % h]);
            const cd even = 0.5 * (zk + zc);
            const cd odd = cd(0, -0.5) * (zk - zc);
            X[k] = even + w[k] * odd;
        }
    }
};

enum Kind { C2C, R2C, C2R, R2R };

struct Plan {
    Kind kind;
    int rank;
    int n[2];
    int howmany;
    int inembed[2], onembed[2];
    int istride, idist, ostride, odist;
    int sign;
    int r2rKind[2];
    void* in;
    void* out;
    std::vector<std::unique_ptr<Fft1d>> fwd; /* per dimension, sign as planned */
    std::unique_ptr<Rfft1d> rfft;             /* last dimension, for R2C */
    std::unique_ptr<Fft1d> lastInv;           /* last dimension inverse, for C2R */
    std::vector<std::vector<double>> cosTab;  /* per dimension, for R2R */
};

void copyDims(Plan* p, int rank, const int* n, const int* inembed, const int* onembed, bool r2cOut, bool c2rIn) {
    p->rank = rank;
    for (int d = 0; d < 2; d++) { p->n[d] = 1; p->inembed[d] = 1; p->onembed[d] = 1; }
    for (int d = 0; d < rank; d++) p->n[d] = n[d];
    for (int d = 0; d < rank; d++) {
        int ni = n[d], no = n[d];
        if (d == rank - 1 && r2cOut) no = n[d] / 2 + 1;
        if (d == rank - 1 && c2rIn) ni = n[d] / 2 + 1;
        p->inembed[d] = inembed ? inembed[d] : ni;
        p->onembed[d] = onembed ? onembed[d] : no;
    }
}

/* index of element (i0, i1) in an embedded rank-1/2 array */
inline size_t at(const Plan* p, bool input, int i0, int i1) {
    if (p->rank == 1) return (size_t)i0 * (input ? p->istride : p->ostride);
    const int inner = input ? p->inembed[1] : p->onembed[1];
    return ((size_t)i0 * inner + i1) * (size_t)(input ? p->istride : p->ostride);
}

/* Complex transform over rows (last dim) then columns. buf holds n0 x n1 doubles-complex. */
void c2cInPlace(const Plan* p, std::vector<cd>& buf, const std::vector<std::unique_ptr<Fft1d>>& f) {
    const int n0 = p->rank == 2 ? p->n[0] : 1;
    const int n1 = p->rank == 2 ? p->n[1] : p->n[0];
    std::vector<cd> tmp((size_t)(n0 > n1 ? n0 : n1));
    const Fft1d& fl = *f[p->rank - 1];
    for (int r = 0; r < n0; r++) {
        fl.run(&buf[(size_t)r * n1], 1, tmp.data());
        std::memcpy(&buf[(size_t)r * n1], tmp.data(), sizeof(cd) * n1);
    }
    if (p->rank == 2) {
        const Fft1d& f0 = *f[0];
        for (int c = 0; c < n1; c++) {
            f0.run(&buf[c], (size_t)n1, tmp.data());
            for (int r = 0; r < n0; r++) buf[(size_t)r * n1 + c] = tmp[r];
        }
    }
}

void execC2C(const Plan* p, const fftwf_complex* in, fftwf_complex* out) {
    const int n0 = p->rank == 2 ? p->n[0] : 1;
    const int n1 = p->rank == 2 ? p->n[1] : p->n[0];
    std::vector<cd> buf((size_t)n0 * n1);
    for (int b = 0; b < p->howmany; b++) {
        const fftwf_complex* ib = in + (size_t)b * p->idist;
        fftwf_complex* ob = out + (size_t)b * p->odist;
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++) {
                const size_t s = p->rank == 2 ? at(p, true, i, j) : at(p, true, j, 0);
                buf[(size_t)i * n1 + j] = cd(ib[s][0], ib[s][1]);
            }
        c2cInPlace(p, buf, p->fwd);
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++) {
                const size_t s = p->rank == 2 ? at(p, false, i, j) : at(p, false, j, 0);
                ob[s][0] = (float)buf[(size_t)i * n1 + j].real();
                ob[s][1] = (float)buf[(size_t)i * n1 + j].imag();
            }
    }
}

void execR2C(const Plan* p, const float* in, fftwf_complex* out) {
    const int n0 = p->rank == 2 ? p->n[0] : 1;
    const int n1 = p->rank == 2 ? p->n[1] : p->n[0];
    const int h1 = n1 / 2 + 1;
    std::vector<double> row(n1);
    std::vector<cd> buf((size_t)n0 * h1), col(n0), colOut(n0);
    for (int b = 0; b < p->howmany; b++) {
        const float* ib = in + (size_t)b * p->idist;
        fftwf_complex* ob = out + (size_t)b * p->odist;
        for (int r = 0; r < n0; r++) {
            for (int c = 0; c < n1; c++) row[c] = ib[p->rank == 2 ? at(p, true, r, c) : at(p, true, c, 0)];
            if (n1 % 2 == 0) {
                p->rfft->run(row.data(), &buf[(size_t)r * h1]);
            } else {
                std::vector<cd> z(n1), Z(n1);
                for (int c = 0; c < n1; c++) z[c] = row[c];
                p->fwd[p->rank - 1]->run(z.data(), 1, Z.data());
                for (int c = 0; c < h1; c++) buf[(size_t)r * h1 + c] = Z[c];
            }
        }
        if (p->rank == 2) {
            for (int c = 0; c < h1; c++) {
                for (int r = 0; r < n0; r++) col[r] = buf[(size_t)r * h1 + c];
                p->fwd[0]->run(col.data(), 1, colOut.data());
                for (int r = 0; r < n0; r++) buf[(size_t)r * h1 + c] = colOut[r];
            }
        }
        for (int r = 0; r < n0; r++)
            for (int c = 0; c < h1; c++) {
                const size_t s = p->rank == 2 ? at(p, false, r, c) : at(p, false, c, 0);
                ob[s][0] = (float)buf[(size_t)r * h1 + c].real();
                ob[s][1] = (float)buf[(size_t)r * h1 + c].imag();
            }
    }
}

void execC2R(const Plan* p, const fftwf_complex* in, float* out) {
    const int n0 = p->rank == 2 ? p->n[0] : 1;
    const int n1 = p->rank == 2 ? p->n[1] : p->n[0];
    const int h1 = n1 / 2 + 1;
    std::vector<cd> buf((size_t)n0 * h1), col(n0), colOut(n0), full(n1), fullOut(n1);
    for (int b = 0; b < p->howmany; b++) {
        const fftwf_complex* ib = in + (size_t)b * p->idist;
        float* ob = out + (size_t)b * p->odist;
        for (int r = 0; r < n0; r++)
            for (int c = 0; c < h1; c++) {
                const size_t s = p->rank == 2 ? at(p, true, r, c) : at(p, true, c, 0);
                buf[(size_t)r * h1 + c] = cd(ib[s][0], ib[s][1]);
            }
        if (p->rank == 2) {
            for (int c = 0; c < h1; c++) {
                for (int r = 0; r < n0; r++) col[r] = buf[(size_t)r * h1 + c];
                p->fwd[0]->run(col.data(), 1, colOut.data());
                for (int r = 0; r < n0; r++) buf[(size_t)r * h1 + c] = colOut[r];
            }
        }
        for (int r = 0; r < n0; r++) {
            /* rebuild the Hermitian-symmetric row and take the inverse DFT's real part */
            for (int c = 0; c < h1; c++) full[c] = buf[(size_t)r * h1 + c];
            for (int c = h1; c < n1; c++) full[c] = std::conj(buf[(size_t)r * h1 + (n1 - c)]);
            p->lastInv->run(full.data(), 1, fullOut.data());
            for (int c = 0; c < n1; c++) {
                const size_t s = p->rank == 2 ? at(p, false, r, c) : at(p, false, c, 0);
                ob[s] = (float)fullOut[c].real();
            }
        }
    }
}

/* FFTW3 manual definitions (n = logical length):
 * REDFT10: Y_k = 2 sum_j X_j cos(pi (j + 1/2) k / n)
 * REDFT01: Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (k + 1/2) / n) */
void r2r1d(int kind, const std::vector<double>& tab, int n, const double* x, size_t sx, double* y, size_t sy) {
    /* tab[m] = cos(pi m / (2n)), m in [0, 4n) */
    const int period = 4 * n;
    for (int k = 0; k < n; k++) {
        double acc = 0;
        if (kind == FFTW_REDFT10) {
            for (int j = 0; j < n; j++) acc += x[j * sx] * tab[((2 * j + 1) * k) % period];
            acc *= 2.0;
        } else { /* REDFT01 */
            acc = x[0];
            double s = 0;
            for (int j = 1; j < n; j++) s += x[j * sx] * tab[(j * (2 * k + 1)) % period];
            acc += 2.0 * s;
        }
        y[k * sy] = acc;
    }
}

void execR2R(const Plan* p, const float* in, float* out) {
    const int n0 = p->n[0], n1 = p->n[1];
    std::vector<double> a((size_t)n0 * n1), b((size_t)n0 * n1);
    for (size_t i = 0; i < a.size(); i++) a[i] = in[i];
    for (int r = 0; r < n0; r++) r2r1d(p->r2rKind[1], p->cosTab[1], n1, &a[(size_t)r * n1], 1, &b[(size_t)r * n1], 1);
    for (int c = 0; c < n1; c++) r2r1d(p->r2rKind[0], p->cosTab[0], n0, &b[c], (size_t)n1, &a[c], (size_t)n1);
    for (size_t i = 0; i < a.size(); i++) out[i] = (float)a[i];
}

std::vector<double> makeCosTab(int n) {
    std::vector<double> t((size_t)4 * n);
    for (int m = 0; m < 4 * n; m++) t[m] = std::cos(kPi * (double)m / (2.0 * n));
    return t;
}

} // namespace

struct fftwf_plan_s : public Plan {};

extern "C" {

int fftwf_init_threads(void) { return 1; }
/* Each execute runs on the calling thread; the reference parallelises over
 * frames with its own pool when batchCount > 1 (digHolo.cpp:6993-7038). */
void fftwf_plan_with_nthreads(int) {}

fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany,
                               fftwf_complex* in, const int* inembed, int istride, int idist,
                               fftwf_complex* out, const int* onembed, int ostride, int odist,
                               int sign, unsigned) {
    if (rank < 1 || rank > 2) return nullptr;
    fftwf_plan p = new fftwf_plan_s();
    p->kind = C2C;
    copyDims(p, rank, n, inembed, onembed, false, false);
    p->howmany = howmany; p->istride = istride; p->idist = idist; p->ostride = ostride; p->odist = odist;
    p->sign = sign; p->in = in; p->out = out;
    for (int d = 0; d < rank; d++) p->fwd.emplace_back(new Fft1d(n[d], sign));
    return p;
}

fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                   float* in, const int* inembed, int istride, int idist,
                                   fftwf_complex* out, const int* onembed, int ostride, int odist,
                                   unsigned) {
    if (rank < 1 || rank > 2) return nullptr;
    fftwf_plan p = new fftwf_plan_s();
    p->kind = R2C;
    copyDims(p, rank, n, inembed, onembed, true, false);
    p->howmany = howmany; p->istride = istride; p->idist = idist; p->ostride = ostride; p->odist = odist;
    p->sign = FFTW_FORWARD; p->in = in; p->out = out;
    for (int d = 0; d < rank; d++) p->fwd.emplace_back(new Fft1d(n[d], FFTW_FORWARD));
    if (n[rank - 1] % 2 == 0) p->rfft.reset(new Rfft1d(n[rank - 1]));
    return p;
}

fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                   fftwf_complex* in, const int* inembed, int istride, int idist,
                                   float* out, const int* onembed, int ostride, int odist,
                                   unsigned) {
    if (rank < 1 || rank > 2) return nullptr;
    fftwf_plan p = new fftwf_plan_s();
    p->kind = C2R;
    copyDims(p, rank, n, inembed, onembed, false, true);
    p->howmany = howmany; p->istride = istride; p->idist = idist; p->ostride = ostride; p->odist = odist;
    p->sign = FFTW_BACKWARD; p->in = in; p->out = out;
    for (int d = 0; d < rank; d++) p->fwd.emplace_back(new Fft1d(n[d], FFTW_BACKWARD));
    p->lastInv.reset(new Fft1d(n[rank - 1], FFTW_BACKWARD));
    return p;
}

fftwf_plan fftwf_plan_r2r_2d(int n0, int n1, float* in, float* out,
                             fftwf_r2r_kind kind0, fftwf_r2r_kind kind1, unsigned) {
    fftwf_plan p = new fftwf_plan_s();
    p->kind = R2R;
    p->rank = 2; p->n[0] = n0; p->n[1] = n1; p->howmany = 1;
    p->r2rKind[0] = kind0; p->r2rKind[1] = kind1;
    p->in = in; p->out = out;
    p->cosTab.push_back(makeCosTab(n0));
    p->cosTab.push_back(makeCosTab(n1));
    return p;
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out) {
    if (p && p->kind == C2C) execC2C(p, in, out);
}
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out) {
    if (p && p->kind == R2C) execR2C(p, in, out);
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out) {
    if (p && p->kind == C2R) execC2R(p, in, out);
}
void fftwf_execute_r2r(const fftwf_plan p, float* in, float* out) {
    if (p && p->kind == R2R) execR2R(p, in, out);
}
void fftwf_execute(const fftwf_plan p) {
    if (!p) return;
    switch (p->kind) {
    case C2C: execC2C(p, (fftwf_complex*)p->in, (fftwf_complex*)p->out); break;
    case R2C: execR2C(p, (float*)p->in, (fftwf_complex*)p->out); break;
    case C2R: execC2R(p, (fftwf_complex*)p->in, (float*)p->out); break;
    case R2R: execR2R(p, (float*)p->in, (float*)p->out); break;
    }
}
void fftwf_destroy_plan(fftwf_plan p) { delete p; }

int fftwf_import_wisdom_from_filename(const char*) { return 0; }
int fftwf_export_wisdom_to_filename(const char*) { return 1; }
void fftwf_forget_wisdom(void) {}

} // extern "C"
