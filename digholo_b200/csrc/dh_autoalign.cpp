// Power meter (IL, MDL and the cross-talk metrics) and the AutoAlign
// coordinate search, restated from digHoloPowerMeter (digHolo.cpp:10714-11130),
// digHoloPowerMeterThreaded (digHolo.cpp:12101-12196) and AutoAlign
// (digHolo.cpp:12237-12982) for a single wavelength.  Every evaluation runs
// the GPU batch path; the metric matrices, their FP64 Gram matrices and the
// eigenvalues behind MDL are computed on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dh_object.h"

struct DhEigen;
cudaError_t dh_launch_gather_block(const float2* src0, const float2* src1, int pol0, int pol1, int polCount, int M,
                                   int rows, int batch, float2* A, cudaStream_t s);
cudaError_t dh_launch_gram(const float2* A, int rows, int batch, int rowsGram, void* G, cudaStream_t s);
int dh_eigen_extremes(DhEigen& e, void* G, int n, int count, double* W, void* vecs, double* trace, cudaStream_t s);
DhEigen* dh_eigen_create();
cudaError_t dh_launch_mdl_weights(const float2* A, int rows, int batch, int rowsGram, const double2* u, double alpha,
                                  int pol0, int pol1, int polCount, int M, float2* W, cudaStream_t s);

namespace dh {

static const float PI_F = 3.14159265358979323846264338327950288f;
static const float UNIT_ANGLE = PI_F / 180.0f;
enum { AA_WAIST = 0, AA_DEFOCUS = 1, AA_TILTX = 2, AA_CX = 3, AA_TILTY = 4, AA_CY = 5 };  // digHolo.cpp:2938-2943

static int hgGroup(int mode) {
    int g = 0;
    while ((g + 1) * (g + 2) / 2 <= mode) g++;
    return g;  // m + n of the mode
}

// One matrix block of the power meter: rows = modes (M or 2M), cols = batch.
struct Block {
    const float2* src0;
    const float2* src1;
    int pol0, pol1, rows;
};

// The smallest and largest squared singular value of a block and the sum of
// all of them (its squared Frobenius norm), via the extreme eigenvalues and
// the trace of its smaller Gram matrix.
static int blockSingular2(Object& o, const Block& blk, double& s2min, double& s2max, double& s2sum) {
    const int B = o.batchCount, M = objOutputModes(o), P = o.polCount;
    const size_t aBytes = (size_t)blk.rows * B * sizeof(float2);
    const int rowsGram = blk.rows <= B;
    const int n = rowsGram ? blk.rows : B;
    if (o.dMetricA.ensure(aBytes) != cudaSuccess) return ERR_MEMORYALLOCATION;
    if (o.dMetricG.ensure((size_t)n * n * 16 + (size_t)(n + 1) * sizeof(double)) != cudaSuccess) return ERR_MEMORYALLOCATION;
    if (dh_launch_gather_block(blk.src0, blk.src1, blk.pol0, blk.pol1, P, M, blk.rows, B, o.dMetricA.as<float2>(),
                               o.stream) != cudaSuccess) return ERR_ERROR;
    if (dh_launch_gram(o.dMetricA.as<float2>(), blk.rows, B, rowsGram, o.dMetricG.ptr, o.stream) != cudaSuccess) return ERR_ERROR;
    double* W = reinterpret_cast<double*>(o.dMetricG.as<char>() + (size_t)n * n * 16);   // [n] + trace
    if (!o.eigen) o.eigen = dh_eigen_create();
    if (dh_eigen_extremes(*o.eigen, o.dMetricG.ptr, n, 1, W, nullptr, W + n, o.stream)) return ERR_ERROR;
    double h[3];
    if (cudaMemcpyAsync(&h[0], W, sizeof(double), cudaMemcpyDeviceToHost, o.stream) != cudaSuccess ||
        cudaMemcpyAsync(&h[1], W + n - 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, o.stream) != cudaSuccess)
        return ERR_ERROR;
    if (cudaStreamSynchronize(o.stream) != cudaSuccess) return ERR_ERROR;
    s2min = h[0] < 0 ? 0 : h[0];
    s2max = h[1] < 0 ? 0 : h[1];
    s2sum = h[2] < 0 ? 0 : h[2];
    return ERR_SUCCESS;
}

// MDL of the batch (the power meter's SVD path, digHolo.cpp:11012-11062,
// over all polarisations: blocks as powerMeter forms them) and the weights
// of its gradient: W[frame][pol M + mode] such that
//   d MDL_dB = 20 / ln 10 * Re sum W dc,
// W = w_min / lambda_min - w_max / lambda_max, w of an eigenpair of the
// block Gram matrix as dh_launch_mdl_weights forms it (lambda_min and
// lambda_max the extremes over all blocks, from the FP64 eigensolver with
// their eigenvectors).  Coefficients in the HG basis (the overlap's).
int objMdlWeights(Object& o, float2* W, double* mdlDb) {
    const int B = o.batchCount, P = o.polCount, M = o.modeCount;
    const float2* coefs = o.dCoefs.as<float2>();
    if (M <= 0 || !coefs || B < 1) return ERR_NULLPOINTER;
    const bool indep = o.cfg.autoAlignPolIndependence || P == 1;
    std::vector<Block> blocks;
    if (P == 1) blocks.push_back({coefs, coefs, 0, 0, M});
    else if (indep) { blocks.push_back({coefs, coefs, 0, 0, M}); blocks.push_back({coefs, coefs, 1, 1, M}); }
    else blocks.push_back({coefs, coefs, 0, 1, 2 * M});
    const int rows = blocks[0].rows, K = (int)blocks.size();
    const int rowsGram = rows <= B;
    const int n = rowsGram ? rows : B;
    const size_t aElems = (size_t)rows * B;
    if (o.dMetricA.ensure((size_t)K * aElems * sizeof(float2)) != cudaSuccess) return ERR_MEMORYALLOCATION;
    const size_t gBytes = (size_t)K * n * n * 16, wBytes = (size_t)K * n * sizeof(double), vBytes = (size_t)K * 2 * n * 16;
    if (o.dMetricG.ensure(gBytes + wBytes + vBytes) != cudaSuccess) return ERR_MEMORYALLOCATION;
    char* gb = o.dMetricG.as<char>();
    double* dW = reinterpret_cast<double*>(gb + gBytes);
    double2* dV = reinterpret_cast<double2*>(gb + gBytes + wBytes);
    if (!o.eigen) o.eigen = dh_eigen_create();
    std::vector<double> ev((size_t)K * n);
    for (int k = 0; k < K; k++) {
        float2* A = o.dMetricA.as<float2>() + (size_t)k * aElems;
        const Block& bl = blocks[k];
        if (dh_launch_gather_block(bl.src0, bl.src1, bl.pol0, bl.pol1, P, M, rows, B, A, o.stream) != cudaSuccess) return ERR_ERROR;
        void* Gk = gb + (size_t)k * n * n * 16;
        if (dh_launch_gram(A, rows, B, rowsGram, Gk, o.stream) != cudaSuccess) return ERR_ERROR;
        if (dh_eigen_extremes(*o.eigen, Gk, n, 1, dW + (size_t)k * n, dV + (size_t)k * 2 * n, nullptr, o.stream))
            return ERR_ERROR;
    }
    if (cudaMemcpyAsync(ev.data(), dW, ev.size() * sizeof(double), cudaMemcpyDeviceToHost, o.stream) != cudaSuccess)
        return ERR_ERROR;
    if (cudaStreamSynchronize(o.stream) != cudaSuccess) return ERR_ERROR;
    int kmin = 0, kmax = 0;
    double lmin = DBL_MAX, lmax = -DBL_MAX;
    for (int k = 0; k < K; k++) {
        const double a = std::max(0.0, ev[(size_t)k * n]), b = std::max(0.0, ev[(size_t)k * n + n - 1]);
        if (a < lmin) { lmin = a; kmin = k; }
        if (b > lmax) { lmax = b; kmax = k; }
    }
    if (mdlDb) *mdlDb = (lmin > 0 && lmax > 0) ? 10.0 * std::log10(lmin / lmax) : -DBL_MAX;
    if (cudaMemsetAsync(W, 0, (size_t)B * P * M * sizeof(float2), o.stream) != cudaSuccess) return ERR_ERROR;
    if (!(lmin > 0 && lmax > 0)) return ERR_SUCCESS;   // MDL undefined: zero gradient
    const int sel[2] = {kmin, kmax};
    const double alpha[2] = {1.0 / lmin, -1.0 / lmax};
    for (int t = 0; t < 2; t++) {
        const int k = sel[t];
        const Block& bl = blocks[k];
        if (dh_launch_mdl_weights(o.dMetricA.as<float2>() + (size_t)k * aElems, rows, B, rowsGram,
                                  dV + ((size_t)k * 2 + t) * n, alpha[t], bl.pol0, bl.pol1, P, M, W, o.stream) != cudaSuccess)
            return ERR_ERROR;
    }
    return ERR_SUCCESS;
}

// digHoloPowerMeter for one wavelength.  polIdx < 0: all polarisations.
// `other` (device coefficients) supplies the other polarisation when one
// polarisation is evaluated with non-independent polarisations.
int powerMeter(Object& o, float* out, int polIdx, int polsIndependent, const float2* other, bool doIL, bool doMDL,
               bool doXtalk, bool mulConj) {
    const int B = o.batchCount, P = o.polCount, M = objOutputModes(o);
    const float2* coefs = objOutputCoefs(o);
    float il = 0.f, mdl = 0.f;
    for (int i = 0; i < METRIC_COUNT; i++) out[i] = 0.f;
    if (M <= 0 || !coefs) return ERR_NULLPOINTER;
    // host copy of the coefficients for the element-wise metrics
    std::vector<float> hc((size_t)B * P * M * 2);
    if (cudaMemcpyAsync(hc.data(), coefs, hc.size() * sizeof(float), cudaMemcpyDeviceToHost, o.stream) != cudaSuccess)
        return ERR_ERROR;
    std::vector<float> ho;
    const float2* otherSrc = other ? other : coefs;
    if (P == 2 && polIdx >= 0 && !polsIndependent) {
        ho.resize(hc.size());
        if (cudaMemcpyAsync(ho.data(), otherSrc, ho.size() * sizeof(float), cudaMemcpyDeviceToHost, o.stream) != cudaSuccess)
            return ERR_ERROR;
    }
    if (cudaStreamSynchronize(o.stream) != cudaSuccess) return ERR_ERROR;

    if (B <= 1) {  // digHolo.cpp:11078-11111
        float total = 0.f, diag = 0.f;
        for (int p = 0; p < P; p++)
            for (int m = 0; m < M; m++) {
                const float vr = hc[((size_t)p * M + m) * 2], vi = hc[((size_t)p * M + m) * 2 + 1];
                const float pw = vr * vr + vi * vi;
                total += pw;
                if (m == 0) diag += pw;
            }
        out[METRIC_IL] = total;
        out[METRIC_MDL] = 0.f;
        out[METRIC_DIAG] = diag;
        out[METRIC_SNRAVG] = FLT_MAX;
        out[METRIC_DIAGBEST] = diag;
        out[METRIC_DIAGWORST] = diag;
        out[METRIC_SNRBEST] = FLT_MAX;
        out[METRIC_SNRWORST] = FLT_MAX;
        out[METRIC_SNRMG] = FLT_MAX;
        return ERR_SUCCESS;
    }

    // matrix blocks (digHolo.cpp:10771-10912), each element (row j, batch b)
    const bool indep = polsIndependent || P == 1;
    std::vector<Block> blocks;
    int svdM = 0;
    // host view: element(j, b) of block k
    auto hostElem = [&](int k, int j, int b, float& re, float& im) {
        const Block& bl = blocks[k];
        const int Mx = M;
        const float* src;
        int pol, jj;
        if (j < Mx) { src = (bl.src0 == coefs) ? hc.data() : ho.data(); pol = bl.pol0; jj = j; }
        else { src = (bl.src1 == coefs) ? hc.data() : ho.data(); pol = bl.pol1; jj = j - Mx; }
        const size_t i = ((size_t)b * P * Mx + (size_t)pol * Mx + jj) * 2;
        re = src[i];
        im = src[i + 1];
    };
    if (P == 1) {
        blocks.push_back({coefs, coefs, 0, 0, M});
    } else if (polIdx >= 0) {
        if (indep) blocks.push_back({coefs, coefs, polIdx, polIdx, M});
        else blocks.push_back({coefs, otherSrc, polIdx, 1 - polIdx, 2 * M});
    } else {
        if (indep) {
            blocks.push_back({coefs, coefs, 0, 0, M});
            blocks.push_back({coefs, coefs, 1, 1, M});
        } else {
            blocks.push_back({coefs, coefs, 0, 1, 2 * M});
        }
    }
    svdM = blocks[0].rows;
    const int svdN = B;
    const int svdCount = (int)blocks.size();

    float totalSignal = 0, totalNoise = 0, totalSNR = 0, totalSignalMG = 0, totalNoiseMG = 0;
    float minSignal = FLT_MAX, maxSignal = -FLT_MAX, minNoise = FLT_MAX, maxNoise = -FLT_MAX;
    float minSNR = FLT_MAX, maxSNR = -FLT_MAX;
    int totalSignalCount = 1;
    if (doXtalk) {  // digHolo.cpp:10924-11008
        for (int k = 0; k < svdCount; k++) {
            int Mv = svdM, Nv = svdN;
            std::vector<double> uu;
            if (mulConj && svdM >= svdN) {
                // UU = A^H A (batch x batch), digHolo.cpp:3062-3101
                const int n = svdN;
                if (o.dMetricA.ensure((size_t)svdM * B * sizeof(float2)) != cudaSuccess) return ERR_MEMORYALLOCATION;
                if (o.dMetricG.ensure((size_t)n * n * 16 + (size_t)n * 8) != cudaSuccess) return ERR_MEMORYALLOCATION;
                const Block& bl = blocks[k];
                if (dh_launch_gather_block(bl.src0, bl.src1, bl.pol0, bl.pol1, P, M, bl.rows, B, o.dMetricA.as<float2>(),
                                           o.stream) != cudaSuccess) return ERR_ERROR;
                if (dh_launch_gram(o.dMetricA.as<float2>(), bl.rows, B, 0, o.dMetricG.ptr, o.stream) != cudaSuccess) return ERR_ERROR;
                uu.resize((size_t)n * n * 2);
                if (cudaMemcpyAsync(uu.data(), o.dMetricG.ptr, uu.size() * sizeof(double), cudaMemcpyDeviceToHost, o.stream) != cudaSuccess)
                    return ERR_ERROR;
                if (cudaStreamSynchronize(o.stream) != cudaSuccess) return ERR_ERROR;
                Mv = svdN;
                Nv = svdN;
            } else if (mulConj) {
                Mv = svdM;
                Nv = svdM;
            }
            totalSignalCount = Mv * Nv * svdCount;
            for (int i = 0; i < Nv && i < M; i++) {
                float signal = 0, noise = 0;
                const int MGin = hgGroup(i) + 1;
                for (int j = 0; j < Mv; j++) {
                    const int MGout = hgGroup(j % M) + 1;
                    float vr, vi;
                    if (!uu.empty()) {
                        // column-major n x n: element (j, i) at i * n + j
                        vr = (float)uu[((size_t)i * Nv + j) * 2];
                        vi = (float)uu[((size_t)i * Nv + j) * 2 + 1];
                    } else if (i < svdN && j < svdM) {
                        hostElem(k, j, i, vr, vi);
                    } else {
                        vr = vi = 0.f;
                    }
                    const float vPwr = vr * vr + vi * vi;
                    if (i == j || i == (j - M)) signal += vPwr;
                    else noise += vPwr;
                    if (MGin == MGout) totalSignalMG += vPwr / MGin;
                    else totalNoiseMG += vPwr / MGin;
                }
                const float SNR = signal / noise;
                totalSignal += signal;
                totalNoise += noise;
                maxSignal = std::max(maxSignal, signal);
                minSignal = std::min(minSignal, signal);
                maxNoise = std::max(maxNoise, noise);
                minNoise = std::min(minNoise, noise);
                if (SNR < minSNR) minSNR = SNR;
                if (SNR > maxSNR) maxSNR = SNR;
            }
        }
        totalSNR = totalSignal / totalNoise;
    }
    if (doMDL) {  // digHolo.cpp:11012-11062
        // IL: the mean squared singular value (the trace of the Gram matrix
        // over its size); MDL: the smallest over the largest, over all blocks
        const int minDim = std::min(svdM, svdN);
        double sum = 0.0;
        float maxS = -FLT_MAX, minS = FLT_MAX;
        for (int k = 0; k < svdCount; k++) {
            double lo2 = 0.0, hi2 = 0.0, sum2 = 0.0;
            const int r = blockSingular2(o, blocks[k], lo2, hi2, sum2);
            if (r) return r;
            sum += sum2;
            minS = std::min(minS, (float)std::sqrt(lo2));
            maxS = std::max(maxS, (float)std::sqrt(hi2));
        }
        il = (float)(sum / ((double)svdCount * minDim));
        mdl = (minS * minS) / (maxS * maxS);
    } else if (doIL) {  // insertionLoss256, digHolo.cpp:3105-3143
        il = 0.f;
        for (int k = 0; k < svdCount; k++) {
            double acc = 0.0;
            for (int b = 0; b < svdN; b++)
                for (int j = 0; j < svdM; j++) {
                    float vr, vi;
                    hostElem(k, j, b, vr, vi);
                    acc += (double)vr * vr + (double)vi * vi;
                }
            il += (float)(acc / svdN);
        }
    }
    out[METRIC_IL] = il;
    out[METRIC_MDL] = mdl;
    out[METRIC_DIAG] = totalSignal / totalSignalCount;
    out[METRIC_SNRAVG] = totalSNR;
    out[METRIC_DIAGBEST] = maxSignal;
    out[METRIC_DIAGWORST] = minSignal;
    out[METRIC_SNRBEST] = maxSNR;
    out[METRIC_SNRWORST] = minSNR;
    out[METRIC_SNRMG] = totalSignalMG / totalNoiseMG;
    return ERR_SUCCESS;
}

// digHoloPowerMeterThreaded for one wavelength: linear metrics to dB
// (entries [metric][0] and the average [metric][1] are equal).
static int powerMeterDB(Object& o, float out[][METRIC_COUNT], int polThreads, int polsIndependent, const float2* backup,
                        bool doIL, bool doMDL, bool doXtalk, bool mulConj) {
    for (int t = 0; t < polThreads; t++) {
        const int r = powerMeter(o, out[t], polThreads == 2 ? t : -1, polsIndependent, backup, doIL, doMDL, doXtalk, mulConj);
        if (r) return r;
        for (int m = 0; m < METRIC_COUNT; m++) out[t][m] = 10.f * log10f(out[t][m]);
    }
    return ERR_SUCCESS;
}

int objCalcMetrics(Object& o) {
    if (!o.processedOverlap || o.modeCount <= 0) return ERR_NULLPOINTER;
    float out[2][METRIC_COUNT];
    const int r = powerMeterDB(o, out, 1, o.cfg.autoAlignPolIndependence, nullptr, true, true, true,
                               o.cfg.autoAlignBasisMulConjTrans != 0);
    if (r) return r;
    for (int m = 0; m < METRIC_COUNT; m++) o.autoAlignMetrics[m][0] = o.autoAlignMetrics[m][1] = out[0][m];
    o.metricsValid = 1;
    return ERR_SUCCESS;
}

// ------------------------------------------------------------- AutoAlign

static float aaGet(const Config& c, int pol, int par) {
    switch (par) {
        case AA_TILTX: return c.zern[pol][ZERN_TILTX];
        case AA_TILTY: return c.zern[pol][ZERN_TILTY];
        case AA_CX: return c.beamCentreX[pol];
        case AA_CY: return c.beamCentreY[pol];
        case AA_DEFOCUS: return c.zern[pol][ZERN_DEFOCUS];
        case AA_WAIST: return c.waist[pol];
    }
    return -FLT_MAX;
}
static void aaSet(Config& c, int pol, int par, float v) {
    switch (par) {
        case AA_TILTX: c.zern[pol][ZERN_TILTX] = v; break;
        case AA_TILTY: c.zern[pol][ZERN_TILTY] = v; break;
        case AA_CX: c.beamCentreX[pol] = v; break;
        case AA_CY: c.beamCentreY[pol] = v; break;
        case AA_DEFOCUS: c.zern[pol][ZERN_DEFOCUS] = v; break;
        case AA_WAIST: c.waist[pol] = v; break;
    }
}
static void alignmentSave(const Config& c, int pol, float* s) {
    for (int par = 0; par < 6; par++) s[par] = aaGet(c, pol, par);
}
static void alignmentLoad(Config& c, int pol, const float* s) {
    for (int par = 0; par < 6; par++) aaSet(c, pol, par, s[par]);
}

// FourierWindowRadiusMax / Rec (digHolo.cpp:11964-11993)
static float windowRadiusMax(float pixelSize, float wavelength) {
    const float wc = (float)((-2.0 + std::sqrt(68.0)) / 16.0);
    const float wmax = (float)(wavelength / (2.0 * pixelSize));
    return (wc * wmax) / UNIT_ANGLE;
}
static float windowRadiusRec(const Config& c, int P) {
    float tMin = FLT_MAX;
    for (int p = 0; p < P; p++) {
        const float tx = c.zern[p][ZERN_TILTX], ty = c.zern[p][ZERN_TILTY];
        tMin = std::min(tMin, std::sqrt(tx * tx + ty * ty));
    }
    return tMin / 3.0f;
}

// fitToQuadratic (digHolo.cpp:3146-3252): Gauss-Newton fit of y = a x^2 + b x + c
// from B0, with the normal equations of the 3-parameter linear least squares
// solved directly; returns the vertex -b / 2a (NaN if the data are not finite).
float fitToQuadratic(const float* x, const float* y, int n, float* B, const float* B0, float tol, float maxIter) {
    double a = B0[0], b = B0[1], c = B0[2];
    float resid = 0.f, lastResid = 0.f;
    int iter = 0;
    float maxPoint = 0.f;
    while (true) {
        bool valid = true;
        double JtJ[3][3] = {{0}}, Jtr[3] = {0};
        for (int i = 0; i < n; i++) {
            const float xi = x[i];
            const float jr0 = xi * xi;
            const float yy = (float)(a * xi * xi + b * xi + c);
            const float r = y[i] - yy;
            if (std::isnan(jr0) || std::isnan(r)) valid = false;
            const double J[3] = {jr0, xi, 1.0};
            for (int p = 0; p < 3; p++) {
                Jtr[p] += J[p] * r;
                for (int q = 0; q < 3; q++) JtJ[p][q] += J[p] * J[q];
            }
            resid += r * r;
        }
        if (!valid) return NAN;
        // least-squares step: solve JtJ d = Jtr (3x3, Gaussian elimination with pivoting)
        double Mx[3][4];
        for (int p = 0; p < 3; p++) { for (int q = 0; q < 3; q++) Mx[p][q] = JtJ[p][q]; Mx[p][3] = Jtr[p]; }
        for (int col = 0; col < 3; col++) {
            int piv = col;
            for (int r2 = col + 1; r2 < 3; r2++) if (std::fabs(Mx[r2][col]) > std::fabs(Mx[piv][col])) piv = r2;
            for (int q = 0; q < 4; q++) std::swap(Mx[col][q], Mx[piv][q]);
            if (Mx[col][col] == 0) return NAN;
            for (int r2 = col + 1; r2 < 3; r2++) {
                const double f = Mx[r2][col] / Mx[col][col];
                for (int q = col; q < 4; q++) Mx[r2][q] -= f * Mx[col][q];
            }
        }
        double d[3];
        for (int p = 2; p >= 0; p--) {
            double acc = Mx[p][3];
            for (int q = p + 1; q < 3; q++) acc -= Mx[p][q] * d[q];
            d[p] = acc / Mx[p][p];
        }
        a += d[0]; b += d[1]; c += d[2];
        B[0] = (float)a; B[1] = (float)b; B[2] = (float)c;
        iter++;
        const bool done = std::fabs(resid - lastResid) < tol || iter > maxIter;
        lastResid = resid;
        maxPoint = -B[1] / (2 * B[0]);
        if (done) break;
    }
    return maxPoint;
}


int objAutoAlignSnap(Object& o, float steps[4]);

// AutoAlign (digHolo.cpp:12237-12982), single wavelength.  FULL and
// ESTIMATE start with the parameter estimate (objAutoAlignSnap, dh_snap.cpp);
// ESTIMATE then scores the estimate, FULL and TWEAK refine the settings with
// the reference's coordinate search.
float objAutoAlign(Object& o) {
    Config& c = o.cfg;
    const int P = c.polCount;
    const int goalIdx0 = c.autoAlignGoalIdx;
    const int polsIndependent = c.autoAlignPolIndependence;
    const float tol = c.autoAlignTol;
    const bool mulConj = c.autoAlignBasisMulConjTrans != 0;
    const int maxMG = c.maxMG;
    if (c.autoAlignFourierWindowRadius) {
        c.apertureSize = c.autoAlignTilt ? windowRadiusMax(c.pixelSize, c.wavelengthCentre) : windowRadiusRec(c, P);
    }
    // FULL (0) and ESTIMATE (2): the parameter estimate first, which also
    // sets the step sizes of the search (digHolo.cpp:12301-12314)
    const int mode = c.autoAlignMode;
    float snapSteps[4] = {0.f, 0.f, 0.f, 0.f};
    const bool snapped = mode == 0 || mode == 2 || maxMG <= 0;
    if (snapped) {
        if (objAutoAlignSnap(o, snapSteps)) return -FLT_MAX;
        if (mode == 2 || maxMG <= 0) {
            // the estimate scored by a final overlap and power meter
            // (digHolo.cpp:11925-11953, 12962-12980); this build scores it
            // on the configured FFT window
            if (maxMG <= 0) return -FLT_MAX;
            if (objProcessBatch(o, 0) || objCalcMetrics(o)) return -FLT_MAX;
            return o.autoAlignMetrics[goalIdx0 >= 0 && goalIdx0 < METRIC_COUNT ? goalIdx0 : 0][0];
        }
    }
    // step sizes (digHolo.cpp:12298-12313)
    float tiltStep = c.apertureSize * 0.1f;
    float centreStep = c.waist[0] * 0.1f;
    float defocusStep = 0.4f;
    for (int i = 0; i < P; i++) defocusStep = std::max(defocusStep, std::fabs(c.zern[i][ZERN_DEFOCUS]) * 0.1f);
    float waistStep = c.waist[0] * 0.1f;
    if (snapped) {
        tiltStep = snapSteps[0];
        centreStep = snapSteps[1];
        defocusStep = snapSteps[2];
        waistStep = snapSteps[3];
    }
    if (maxMG <= 0) return -FLT_MAX;

    float LIMS[6][2];
    const float pixel = c.pixelSize;
    LIMS[AA_TILTX][0] = 0;
    LIMS[AA_TILTX][1] = (c.wavelengthCentre / (2 * pixel)) / UNIT_ANGLE;
    LIMS[AA_TILTY][0] = -(c.apertureSize + LIMS[AA_TILTX][1]);
    LIMS[AA_TILTY][1] = (c.apertureSize + LIMS[AA_TILTX][1]);
    LIMS[AA_DEFOCUS][0] = -100;
    LIMS[AA_DEFOCUS][1] = 100;
    LIMS[AA_WAIST][0] = pixel / 3;
    LIMS[AA_WAIST][1] = pixel * (float)std::max(c.frameHeight, c.frameWidth);
    LIMS[AA_CX][0] = -(c.frameWidth / 2.0f) * pixel;
    LIMS[AA_CX][1] = (c.frameWidth / 2.0f) * pixel;
    LIMS[AA_CY][0] = -(c.frameHeight / 2.0f) * pixel;
    LIMS[AA_CY][1] = (c.frameHeight / 2.0f) * pixel;

    const int sampleCount = 3, stepCount = sampleCount + 2;
    float x[2][stepCount + 2], y[2][stepCount + 2], Bq[2][3], B0[2][3];
    float dTxs[stepCount + 2][2];
    float best[2][6];
    alignmentSave(c, 0, best[0]);
    alignmentSave(c, 1, best[1]);
    float stepSize[6];
    stepSize[AA_TILTX] = stepSize[AA_TILTY] = tiltStep;
    stepSize[AA_DEFOCUS] = defocusStep;
    stepSize[AA_CX] = stepSize[AA_CY] = centreStep;
    stepSize[AA_WAIST] = waistStep;
    float stepBounds[6];
    for (int i = 0; i < 6; i++) stepBounds[i] = stepSize[i] * 10;
    const float fitTol = 1e-6f, fitIter = 101;
    const int goalCount = goalIdx0 ? 2 : 1;
    float lastErrTol = goalIdx0 ? 0.1f + tol * 10.0f : tol;
    const int maxAttempts = 20;
    const bool tiltLock = c.polLockTilt, waistLock = c.polLockBasisWaist, defocusLock = c.polLockDefocus;
    float out[2][METRIC_COUNT], outBest[2][METRIC_COUNT], outf[2][METRIC_COUNT];
    // Frames from host memory are copied to the device once for the whole search.
    const void* userFrames = o.frames;
    const int userOnDevice = o.framesOnDevice;
    struct Restore {
        Object& o; const void* f; int d;
        ~Restore() { o.frames = f; o.framesOnDevice = d; o.preparedValid = 0; o.useSnaps = 0; }
    } restore{o, userFrames, userOnDevice};
    // Stage semantics of the reference's search: the FFT runs once (first
    // evaluation), the IFFT (Fourier-window selection) reruns only when the
    // beam centre changes and after each parameter, and the tilt removal and
    // overlap rerun for every evaluation (digHolo.cpp:12599-12645, 12795-12802).
    o.useSnaps = 1;
    o.fftSnap = c;
    o.ifftSnap = c;
    {
        int r0 = objProcessForAlign(o);  // resolves the frame source and the geometry
        if (r0) return -FLT_MAX;
        if (!o.framesOnDevice) {
            const size_t bytes = (size_t)o.batchCount * std::max(1, o.avgCount) * c.frameWidth * c.frameHeight * (o.framesU16 ? 2 : 4);
            if (o.dAlignFrames.ensure(bytes) != cudaSuccess) return -FLT_MAX;
            if (cudaMemcpy(o.dAlignFrames.ptr, o.frames, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return -FLT_MAX;
            o.frames = o.dAlignFrames.ptr;
            o.framesOnDevice = 1;
        }
    }
    // device copy of the best coefficients so far (the other polarisation's
    // matrix half when the polarisations are not independent), taken from the
    // first evaluation as digHolo.cpp:12617-12620 does
    const size_t coefBytes = (size_t)o.batchCount * o.polCount * objOutputModes(o) * sizeof(float2);
    if (o.dCoefsBackup.ensure(coefBytes) != cudaSuccess) return -FLT_MAX;
    const float2* backup = o.dCoefsBackup.as<float2>();
    bool firstRun = true;
    int r = 0;
    o.alignEvaluations = 0;

    for (int goalIDX = 0; goalIDX < goalCount; goalIDX++) {
        const int goalIdx = goalIDX ? goalIdx0 : 0;
        bool converged = false;
        float bestPwr[2] = {-FLT_MAX, -FLT_MAX};
        float lastErr[2] = {FLT_MAX, FLT_MAX};
        outBest[0][goalIdx] = outBest[1][goalIdx] = -FLT_MAX;
        const bool doIL = goalIdx == 0, doMDL = goalIdx == 1, doXtalk = goalIdx >= 2;
        int attempt = 0;
        if (goalIDX) {
            stepSize[AA_TILTX] = stepSize[AA_TILTY] = tiltStep / 10.0f;
            stepSize[AA_DEFOCUS] = defocusStep / 10.0f;
            stepSize[AA_CX] = stepSize[AA_CY] = centreStep / 10.0f;
            stepSize[AA_WAIST] = waistStep / 10.0f;
            lastErrTol = tol;
        }
        while (!converged) {
            bool enabled[6];
            enabled[AA_TILTX] = enabled[AA_TILTY] = c.autoAlignTilt;
            enabled[AA_CX] = enabled[AA_CY] = c.autoAlignCentre;
            enabled[AA_WAIST] = c.autoAlignBasisWaist;
            enabled[AA_DEFOCUS] = c.autoAlignDefocus;
            for (int par = 0; par < 6; par++) {
                if (!enabled[par]) continue;
                const bool lock = ((par == AA_TILTX || par == AA_TILTY) && tiltLock) || (par == AA_DEFOCUS && defocusLock) ||
                                  (par == AA_WAIST && waistLock);
                float var0[2];
                var0[0] = aaGet(c, 0, par);
                var0[1] = lock ? var0[0] : aaGet(c, 1, par);
                float meanPwr[2] = {0, 0}, maxPwr[2] = {-FLT_MAX, -FLT_MAX}, maxima[2] = {0, 0};
                bool isValid[2] = {true, true};
                for (int stepIdx = 0; stepIdx < stepCount + 1; stepIdx++) {
                    float* dTx = dTxs[stepIdx];
                    for (int p = 0; p < P; p++) {
                        if (stepIdx < sampleCount)
                            dTx[p] = (float)(var0[p] + ((stepIdx - (sampleCount - 1) / 2.0) * stepSize[par] / (sampleCount - 1)));
                        if (lock) dTx[1] = dTx[0];
                        if (dTx[p] > LIMS[par][1]) dTx[p] = LIMS[par][1];
                        if (dTx[p] < LIMS[par][0]) dTx[p] = LIMS[par][0];
                        isValid[p] = !std::isnan(dTx[p]) && !std::isinf(dTx[p]);
                        if (isValid[p]) aaSet(c, p, par, dTx[p]);
                    }
                    if (c.autoAlignFourierWindowRadius) {
                        const float apMax = windowRadiusRec(c, P);
                        if (c.apertureSize > apMax) {
                            c.apertureSize = apMax;
                            o.ifftSnap.apertureSize = apMax;   // the working radius follows at once
                        }
                    }
                    if (firstRun) o.fftSnap = c;
                    if (firstRun || par == AA_CX || par == AA_CY) {
                        const float ap = o.ifftSnap.apertureSize;
                        o.ifftSnap = c;
                        o.ifftSnap.apertureSize = ap;
                    }
                    r = objProcessForAlign(o);
                    if (r) return -FLT_MAX;
                    o.alignEvaluations++;
                    if (firstRun) {
                        cudaMemcpyAsync(o.dCoefsBackup.ptr, objOutputCoefs(o), coefBytes, cudaMemcpyDeviceToDevice, o.stream);
                        firstRun = false;
                    }
                    if ((!lock && P > 1) || polsIndependent) {
                        r = powerMeterDB(o, out, 2, polsIndependent, backup, doIL, doMDL, doXtalk, mulConj);
                    } else {
                        r = powerMeterDB(o, out, 1, polsIndependent, backup, doIL, doMDL, doXtalk, mulConj);
                        memcpy(out[1], out[0], sizeof(out[0]));
                    }
                    if (r) return -FLT_MAX;
                    for (int i = 0; i < P; i++) {
                        const float pwr = out[i][goalIdx];
                        x[i][stepIdx] = dTx[i];
                        y[i][stepIdx] = pwr;
                        if (pwr > maxPwr[i] && isValid[i]) {
                            maxPwr[i] = pwr;
                            if (pwr > bestPwr[i]) {
                                alignmentSave(c, i, best[i]);
                                memcpy(outBest[i], out[i], sizeof(out[i]));
                                // keep this polarisation's coefficients as the best so far
                                cudaMemcpy2DAsync(o.dCoefsBackup.as<float2>() + (size_t)i * objOutputModes(o),
                                                  (size_t)o.polCount * objOutputModes(o) * sizeof(float2),
                                                  objOutputCoefs(o) + (size_t)i * objOutputModes(o),
                                                  (size_t)o.polCount * objOutputModes(o) * sizeof(float2),
                                                  (size_t)objOutputModes(o) * sizeof(float2), o.batchCount,
                                                  cudaMemcpyDeviceToDevice, o.stream);
                                bestPwr[i] = pwr;
                            }
                        }
                        meanPwr[i] += pwr;
                        if (stepIdx >= sampleCount - 1) {
                            if (stepIdx == sampleCount - 1) {
                                B0[i][0] = 0;
                                B0[i][1] = 0;
                                B0[i][2] = meanPwr[i] / (stepIdx + 1);
                                for (int s0 = 0; s0 <= stepIdx; s0++)
                                    for (int s1 = 1; s1 <= stepIdx; s1++)
                                        if (y[i][s1] < y[i][s1 - 1]) {
                                            std::swap(y[i][s1], y[i][s1 - 1]);
                                            std::swap(x[i][s1], x[i][s1 - 1]);
                                        }
                            }
                            maxima[i] = fitToQuadratic(x[i], y[i], stepIdx + 1, Bq[i], B0[i], fitTol, fitIter);
                            const bool valid = !std::isnan(maxima[0]) && !std::isinf(maxima[0]);
                            if (valid) {
                                dTxs[stepIdx + 1][i] = maxima[i];
                                const float dBest = maxima[i] - best[i][par];
                                if (std::fabs(dBest) > stepBounds[par])
                                    dTxs[stepIdx + 1][i] = dBest > stepBounds[par] ? best[i][par] + stepBounds[par]
                                                                                   : best[i][par] - stepBounds[par];
                            } else {
                                dTxs[stepIdx + 1][i] = (float)(best[i][par] + ((stepIdx - (stepCount - 1) / 2.0) * stepSize[par] / (stepCount - 1)));
                            }
                            for (int q = 0; q < 3; q++) B0[i][q] = Bq[i][q];
                        }
                    }
                }
                for (int p = 0; p < P; p++) alignmentLoad(c, p, best[p]);
                {
                    const float ap = o.ifftSnap.apertureSize;
                    o.ifftSnap = c;
                    o.ifftSnap.apertureSize = ap;
                }
            }
            r = objProcessForAlign(o);
            if (r) return -FLT_MAX;
            o.alignEvaluations++;
            if (firstRun) {
                cudaMemcpyAsync(o.dCoefsBackup.ptr, objOutputCoefs(o), coefBytes, cudaMemcpyDeviceToDevice, o.stream);
                firstRun = false;
            }
            r = powerMeterDB(o, outf, 1, polsIndependent, nullptr, true, true, true, mulConj);
            if (r) return -FLT_MAX;
            cudaMemcpyAsync(o.dCoefsBackup.ptr, objOutputCoefs(o), coefBytes, cudaMemcpyDeviceToDevice, o.stream);
            float dErr = 0;
            for (int p = 0; p < P; p++) {
                dErr += std::fabs(outBest[p][goalIdx] - lastErr[p]);
                lastErr[p] = outBest[p][goalIdx];
            }
            dErr /= P;
            attempt++;
            if (dErr <= lastErrTol || attempt == maxAttempts) converged = true;
        }
    }
    for (int m = 0; m < METRIC_COUNT; m++) o.autoAlignMetrics[m][0] = o.autoAlignMetrics[m][1] = outf[0][m];
    o.metricsValid = 1;
    objCoefsToHost(o);
    return outf[0][goalIdx0];
}

}  // namespace dh
