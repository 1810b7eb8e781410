// Gradient-driven AutoAlign.  objAlignGradient evaluates the batch path and
// its adjoint on the GPU (dh_align_grad.cu): the gradient of
// IL = 10 log10(sum |c|^2) + const with respect to each polarisation's tilt,
// defocus, beam centre and basis waist, the Fourier-window selection held
// fixed.  objAutoAlignAdjoint maximises the same IL with a quasi-Newton
// (BFGS) iteration in step-normalised coordinates and a backtracking line
// search, in place of the reference's coordinate search (AutoAlign,
// digHolo.cpp:12237-12982), and leaves the metrics of the final
// configuration like digHoloAutoAlign does.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dh_grad.h"
#include "dh_object.h"

namespace dh {

static const double PI_DA = 3.14159265358979323846;
static const float UNIT_ANGLE_A = (float)(PI_DA / 180.0);
enum { G_TX = 0, G_TY = 1, G_DEF = 2, G_CX = 3, G_CY = 4, G_WAIST = 5 };

// grad12[pol * 6 + k], k in {tiltX, tiltY, defocus, beamCentreX, beamCentreY,
// waist} (config units: degrees, dioptre, m, m); parameters tied by the
// polarisation locks carry the sum on polarisation 0 and zero on 1.
// metric 0: IL = 10 log10(S), S = sum |c|^2 (valueOut = IL); metric 1: MDL
// in dB from the extreme eigenvalues of the batch Gram matrix
// (valueOut = MDL), its gradient through the eigenvalue derivatives
// d lambda = u^H dG u (objMdlWeights).
int objAlignGradient(Object& o, float* grad12, float* ilOut) { return objAlignGradientMetric(o, 0, grad12, ilOut); }

int objAlignGradientMetric(Object& o, int metric, float* grad12, float* ilOut) {
    return objAlignEvaluate(o, metric, ALIGN_EVAL_FULL, grad12, ilOut);
}

// stage ALIGN_EVAL_FULL: the batch, the metric and its gradient;
// ALIGN_EVAL_VALUE: the batch and the metric only (grad12 untouched);
// ALIGN_EVAL_GRADIENT: the gradient (and the metric) of the batch state a
// preceding ALIGN_EVAL_VALUE call left on the device, for the same metric.
// The metric is the same number in every stage.
int objAlignEvaluate(Object& o, int metric, int stage, float* grad12, float* ilOut) {
    Config& c = o.cfg;
    if (c.maxMG <= 0) return fail(o, ERR_ERROR, "adjoint AutoAlign needs a modal basis (maxMG > 0)");
    using Clock = std::chrono::steady_clock;
    const auto t0 = Clock::now();
    int r = ERR_SUCCESS;
    if (stage != ALIGN_EVAL_GRADIENT) {
        const int keep = o.keepField32;
        o.keepField32 = 1;
        r = objProcessForAlign(o);
        o.keepField32 = keep;
        if (r) return r;
    }
    const bool valueOnly = stage == ALIGN_EVAL_VALUE;
    const auto t1 = Clock::now();
    const Geometry& g = o.geo;
    if ((g.w & (g.w - 1)) || (g.h & (g.h - 1)))
        return fail(o, ERR_INVALIDDIMENSION, "the adjoint AutoAlign needs power-of-two IFFT window sides on this build");
    if (o.basisActive)
        return fail(o, ERR_INVALIDARGUMENT, "the adjoint AutoAlign works on Hermite-Gaussian coefficients (basis type 0)");
    const int P = o.polCount, B = o.batchCount, G = c.maxMG, M = o.modeCount;
    const int units = B * P;
    const int w = g.w, h = g.h, W = g.W, H = g.H;
    const size_t npix = (size_t)g.nx * g.ny;

    DhGradParams gp;
    memset(&gp, 0, sizeof(gp));
    float2* Vx = nullptr;
    float2* Vy = nullptr;
    float* hx = nullptr;
    float* hy = nullptr;
    auto t2 = t1, t3 = t1;
    if (!valueOnly) {
        // beam-centre phase derivatives of the window: i kx per column, i ky per row
        std::vector<float> tab((size_t)P * (w + h));
        for (int p = 0; p < P; p++) {
            const int sx0 = g.SX[p] - W / 2;
            for (int cc = 0; cc < w; cc++) tab[(size_t)p * w + cc] = g.kx[sx0 + cc];
            for (int j = 0; j < h; j++) {
                int row = (j + g.SY[p] + H / 2) % H;
                if (row < 0) row += H;
                tab[(size_t)P * w + (size_t)p * h + j] = g.ky[row];
            }
        }
        DH_CUDA(o, o.dGradTab.ensure(tab.size() * sizeof(float)));
        DH_CUDA(o, cudaMemcpyAsync(o.dGradTab.ptr, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, o.stream));
        const size_t winElems = (size_t)units * w * h;
        DH_CUDA(o, o.dGradW.ensure(2 * winElems * sizeof(float2)));
        float2* Wx = o.dGradW.as<float2>();
        float2* Wy = Wx + winElems;
        DH_CUDA(o, dh_launch_window_deriv(o.dWindow.as<float2>(), o.dGradTab.as<float>(), o.dGradTab.as<float>() + (size_t)P * w,
                                          w, h, P, units, Wx, Wy, o.stream));
        // fields of the derivative windows
        DH_CUDA(o, o.dGradV.ensure(2 * (size_t)units * npix * sizeof(float2)));
        Vx = o.dGradV.as<float2>();
        Vy = Vx + (size_t)units * npix;
        // both derivative windows in one launch: a batch of 2B frames (Wy follows Wx, Vy follows Vx)
        DH_CUDA(o, o.dGradScratch.ensure(4 * (size_t)units * npix * sizeof(short) + (size_t)7 * P * (2 * B + 1) * sizeof(float)));
        short* sR = o.dGradScratch.as<short>();
        short* sI = sR + 2 * (size_t)units * npix;
        float* sStats = reinterpret_cast<float*>(sI + 2 * (size_t)units * npix);
        r = objInverseAux(o, Wx, 2 * B, Vx, sR, sI, sStats);
        if (r) return r;
        t2 = Clock::now();
        // float modes up to order G + 1 (the waist derivative reaches m + 2)
        const int GE = G + 2;
        const int L = std::max(g.nx, g.ny);
        DH_CUDA(o, o.dGradBasis.ensure((size_t)P * GE * (g.nx + g.ny) * sizeof(float) + (size_t)GE * L * sizeof(short) +
                                       (size_t)GE * sizeof(float)));
        hx = o.dGradBasis.as<float>();
        hy = hx + (size_t)P * GE * g.nx;
        float* scale = hy + (size_t)P * GE * g.ny;
        short* s16 = reinterpret_cast<short*>(scale + GE);
        r = objBasisFloat(o, GE, hx, hy, s16, scale);
        if (r) return r;
        t3 = Clock::now();
    }

    gp.V = o.dField32.as<float2>();
    gp.Vx = Vx;
    gp.Vy = Vy;
    gp.coefs = o.dCoefs.as<float2>();
    gp.hx = hx;
    gp.hy = hy;
    gp.xAxis = o.dX.as<float>();
    gp.yAxis = o.dY.as<float>();
    gp.nx = g.nx;
    gp.ny = g.ny;
    gp.frameCount = B;
    gp.polCount = P;
    gp.G = G;
    gp.M = M;
    const float k0 = (float)(2.0 * PI_DA / c.wavelengthCentre);
    for (int p = 0; p < P; p++) {
        const int st = c.polLockTilt ? 0 : p;
        gp.k0u[p] = k0 * UNIT_ANGLE_A;
        gp.tiltX[p] = c.zern[st][ZERN_TILTX];
        gp.tiltY[p] = c.zern[st][ZERN_TILTY];
        gp.bcx[p] = c.beamCentreX[p];
        gp.bcy[p] = c.beamCentreY[p];
        float wv = c.waist[c.polLockBasisWaist ? 0 : p];
        gp.waist[p] = wv == 0 ? 400e-6f : wv;
    }
    gp.piOverLambda = (float)(PI_DA / c.wavelengthCentre);
    double mdlDb = 0.0;
    if (metric == 1) {
        // the weights of a value stage serve the gradient stage that follows it
        if (stage != ALIGN_EVAL_GRADIENT) {
            DH_CUDA(o, o.dGradWeights.ensure((size_t)units * M * sizeof(float2)));
            r = objMdlWeights(o, o.dGradWeights.as<float2>(), &mdlDb);
            if (r) return fail(o, r, "MDL gradient: eigenvalues of the batch Gram matrix");
            o.alignMdlDb = mdlDb;
        }
        mdlDb = o.alignMdlDb;
        gp.weights = o.dGradWeights.as<float2>();
    }
    DH_CUDA(o, o.dGradOut.ensure((size_t)units * 7 * sizeof(float)));
    gp.out = o.dGradOut.as<float>();
    DH_CUDA(o, valueOnly ? dh_launch_align_power(gp, o.stream) : dh_launch_align_grad(gp, o.stream));
    if (!o.hGradOut.ensure((size_t)units * 7 * sizeof(float))) return fail(o, ERR_MEMORYALLOCATION, "gradient host buffer");
    const float* part = o.hGradOut.as<float>();
    DH_CUDA(o, cudaMemcpyAsync(o.hGradOut.ptr, gp.out, (size_t)units * 7 * sizeof(float), cudaMemcpyDeviceToHost, o.stream));
    const auto t4 = Clock::now();
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    const auto t5 = Clock::now();
    if (c.verbosity >= 3) {
        auto us = [](Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::micro>(b - a).count(); };
        fprintf(stderr, "digholo_b200: gradient host us: batch %.0f, derivative fields %.0f, basis %.0f, adjoint %.0f, wait %.0f\n",
                us(t0, t1), us(t1, t2), us(t2, t3), us(t3, t4), us(t4, t5));
    }
    r = objCheckStatus(o);
    if (r) return r;
    double acc[2][6] = {};
    double S = 0.0;
    for (int u = 0; u < units; u++) {
        for (int k = 0; k < 6; k++) acc[u % P][k] += part[(size_t)u * 7 + k];
        S += part[(size_t)u * 7 + 6];
    }
    // d IL / d theta = 10 / ln 10 * dS / S, dS = 2 Re sum conj(c) dc;
    // d MDL / d theta = 20 / ln 10 * Re sum W dc
    if (ilOut) *ilOut = metric == 1 ? (float)mdlDb : (float)(10.0 * std::log10(S > 0 ? S : 1e-300));
    if (valueOnly) return ERR_SUCCESS;
    const double f = metric == 1 ? 20.0 / std::log(10.0) : ((S > 0) ? 20.0 / std::log(10.0) / S : 0.0);
    for (int p = 0; p < 2; p++)
        for (int k = 0; k < 6; k++) grad12[p * 6 + k] = p < P ? (float)(f * acc[p][k]) : 0.f;
    if (P > 1) {
        auto tie = [&](int k) { grad12[k] += grad12[6 + k]; grad12[6 + k] = 0.f; };
        if (c.polLockTilt) { tie(G_TX); tie(G_TY); }
        if (c.polLockDefocus) tie(G_DEF);
        if (c.polLockBasisWaist) tie(G_WAIST);
    }
    return ERR_SUCCESS;
}

namespace {

struct Param {
    int pol, kind;
    double scale;
};

double getParam(const Config& c, const Param& q) {
    switch (q.kind) {
        case G_TX: return c.zern[q.pol][ZERN_TILTX];
        case G_TY: return c.zern[q.pol][ZERN_TILTY];
        case G_DEF: return c.zern[q.pol][ZERN_DEFOCUS];
        case G_CX: return c.beamCentreX[q.pol];
        case G_CY: return c.beamCentreY[q.pol];
        default: return c.waist[q.pol];
    }
}

void setParam(Config& c, const Param& q, double v) {
    switch (q.kind) {
        case G_TX: c.zern[q.pol][ZERN_TILTX] = (float)v; break;
        case G_TY: c.zern[q.pol][ZERN_TILTY] = (float)v; break;
        case G_DEF: c.zern[q.pol][ZERN_DEFOCUS] = (float)v; break;
        case G_CX: c.beamCentreX[q.pol] = (float)v; break;
        case G_CY: c.beamCentreY[q.pol] = (float)v; break;
        default: c.waist[q.pol] = (float)v; break;
    }
}

// Whether re-selecting the Fourier window with snapshot b gives the batch
// path of snapshot a: the same window geometry and bit-identical window
// factors.  The snapshot's tilt enters the path only through the window's
// position and its mask, and every kernel evaluates the mask with the float32
// steps of windowFactors, so equal factors mean an identical evaluation.
bool sameSelection(const Object& o, const Config& a, const Config& b) {
    Geometry ga, gb;
    fftWindowGeometry(o.fftSnap, o.polCount, ga);
    ifftWindowGeometry(a, o.polCount, ga);
    fftWindowGeometry(o.fftSnap, o.polCount, gb);
    ifftWindowGeometry(b, o.polCount, gb);
    if (ga.W != gb.W || ga.H != gb.H || ga.w != gb.w || ga.h != gb.h || ga.nx != gb.nx || ga.ny != gb.ny) return false;
    for (int p = 0; p < POLMAX; p++)
        if (ga.cx[p] != gb.cx[p] || ga.cy[p] != gb.cy[p] || ga.SX[p] != gb.SX[p] || ga.SY[p] != gb.SY[p]) return false;
    if (ga.kx != gb.kx || ga.ky != gb.ky || ga.x != gb.x || ga.y != gb.y) return false;
    std::vector<float> fa, fb;
    windowFactors(a, o.cfg, ga, o.polCount, fa);
    windowFactors(b, o.cfg, gb, o.polCount, fb);
    return fa.size() == fb.size() && (fa.empty() || memcmp(fa.data(), fb.data(), fa.size() * sizeof(float)) == 0);
}

}  // namespace

// Maximises IL over the enabled alignment parameters (tilt, beam centre,
// defocus, waist; tied polarisations share one parameter).  Each evaluation
// is one GPU batch pass plus its adjoint; the step coordinates are the
// parameters divided by the reference's search step sizes (tilt 0.1 x the
// window radius, centre and waist 0.1 x the waist, defocus 0.4,
// digHolo.cpp:12298-12313).
float objAutoAlignAdjoint(Object& o) {
    Config& c = o.cfg;
    const int P = o.polCount;
    if (c.maxMG <= 0) return -FLT_MAX;
    // frames from host memory go to the device once for the whole search
    const void* userFrames = o.frames;
    const int userOnDevice = o.framesOnDevice;
    struct Restore {
        Object& o; const void* f; int d; int k;
        ~Restore() { o.frames = f; o.framesOnDevice = d; o.keepField32 = k; o.useSnaps = 0; o.preparedValid = 0; }
    } restore{o, userFrames, userOnDevice, o.keepField32};
    o.keepField32 = 1;   // every evaluation needs the float field for the adjoint
    {
        int r0 = objProcessForAlign(o);
        if (r0) return -FLT_MAX;
        if (!o.framesOnDevice) {
            const size_t bytes = (size_t)o.batchCount * std::max(1, o.avgCount) * c.frameWidth * c.frameHeight * (o.framesU16 ? 2 : 4);
            if (o.dAlignFrames.ensure(bytes) != cudaSuccess) return -FLT_MAX;
            if (cudaMemcpy(o.dAlignFrames.ptr, o.frames, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return -FLT_MAX;
            o.frames = o.dAlignFrames.ptr;
            o.framesOnDevice = 1;
        }
    }
    float w0 = c.waist[0] == 0 ? 400e-6f : c.waist[0];
    const double tiltStep = c.apertureSize * 0.1;
    const double centreStep = w0 * 0.1;
    double defocusStep = 0.4;
    for (int p = 0; p < P; p++) defocusStep = std::max(defocusStep, (double)std::fabs(c.zern[p][ZERN_DEFOCUS]) * 0.1);
    const double waistStep = w0 * 0.1;
    std::vector<Param> prm;
    for (int p = 0; p < P; p++) {
        if (c.autoAlignTilt && (p == 0 || !c.polLockTilt)) {
            prm.push_back({p, G_TX, tiltStep});
            prm.push_back({p, G_TY, tiltStep});
        }
        if (c.autoAlignCentre) {
            prm.push_back({p, G_CX, centreStep});
            prm.push_back({p, G_CY, centreStep});
        }
        if (c.autoAlignDefocus && (p == 0 || !c.polLockDefocus)) prm.push_back({p, G_DEF, defocusStep});
        if (c.autoAlignBasisWaist && (p == 0 || !c.polLockBasisWaist)) prm.push_back({p, G_WAIST, waistStep});
    }
    const int n = (int)prm.size();
    o.alignEvaluations = 0;
    std::vector<double> z(n), gz(n), zt(n), gt(n);
    for (int i = 0; i < n; i++) z[i] = getParam(c, prm[i]) / prm[i].scale;
    auto apply = [&](const std::vector<double>& zz) {
        for (int i = 0; i < n; i++) setParam(c, prm[i], zz[i] * prm[i].scale);
        if (c.polLockBasisWaist && P > 1) c.waist[1] = c.waist[0];
    };
    // f = -metric (IL, then MDL for goal MDL; minimised) and its gradient in
    // step coordinates
    int metric = 0;
    // the configuration and window snapshot of the last evaluation (its
    // coefficients are the ones on the device)
    Config lastCfg = c, lastSnap = c;
    bool haveLast = false;
    auto evalF = [&](const std::vector<double>& zz, double& f, std::vector<double>& gg) -> int {
        apply(zz);
        float g12[12], il = 0.f;
        const int r = objAlignGradientMetric(o, metric, g12, &il);
        o.alignEvaluations++;
        haveLast = r == ERR_SUCCESS;
        lastCfg = c;
        lastSnap = o.ifftSnap;
        if (r) return r;
        f = -(double)il;
        for (int i = 0; i < n; i++) gg[i] = -(double)g12[prm[i].pol * 6 + prm[i].kind] * prm[i].scale;
        if (c.verbosity >= 2) {
            fprintf(stderr, "digholo_b200: adjoint AutoAlign evaluation %d: %s %.5f dB, z =", o.alignEvaluations,
                    metric ? "MDL" : "IL", il);
            for (int i = 0; i < n; i++) fprintf(stderr, " %.4f", zz[i]);
            fprintf(stderr, "\n");
        }
        return ERR_SUCCESS;
    };
    // a line-search trial: the batch and the metric only; its gradient
    // (evalG, on the batch state the trial left on the device) only once
    // the trial is accepted
    auto evalV = [&](const std::vector<double>& zz, double& f) -> int {
        apply(zz);
        float il = 0.f;
        const int r = objAlignEvaluate(o, metric, ALIGN_EVAL_VALUE, nullptr, &il);
        o.alignEvaluations++;
        haveLast = r == ERR_SUCCESS;
        lastCfg = c;
        lastSnap = o.ifftSnap;
        if (r) return r;
        f = -(double)il;
        return ERR_SUCCESS;
    };
    auto evalG = [&](std::vector<double>& gg) -> int {
        float g12[12], il = 0.f;
        const int r = objAlignEvaluate(o, metric, ALIGN_EVAL_GRADIENT, g12, &il);
        if (r) return r;
        for (int i = 0; i < n; i++) gg[i] = -(double)g12[prm[i].pol * 6 + prm[i].kind] * prm[i].scale;
        return ERR_SUCCESS;
    };
    // The FFT window stays where the first evaluation put it; the Fourier
    // window selection and mask are held during a round (the gradient
    // assumes them fixed) and re-selected at the reached point between rounds.
    // Within a round the tilts move at most about one Fourier-plane pixel
    // (lambda / (W pixel) radians) from the round's start: beyond that the
    // selection the round holds is no longer the one the tilt implies, and
    // the held-window objective stops describing the batch path.  The best
    // point seen with freshly selected windows is the result.
    o.useSnaps = 1;
    o.fftSnap = o.ifftSnap = c;
    const double tiltTrust = std::max(0.5, (double)(c.wavelengthCentre / (o.geo.W * c.pixelSize)) / UNIT_ANGLE_A / tiltStep);
    std::vector<char> isTilt(n, 0);
    for (int i = 0; i < n; i++) isTilt[i] = prm[i].kind == G_TX || prm[i].kind == G_TY;
    // goal MDL: as the reference's search (digHolo.cpp:12458-12467), a pass
    // on IL first, then one on the goal
    const int passes = c.autoAlignGoalIdx == METRIC_MDL ? 2 : 1;
    for (int pass = 0; pass < passes; pass++) {
        metric = pass ? METRIC_MDL : METRIC_IL;
        double f = 0.0;
        if (n == 0 || evalF(z, f, gz)) {
            objCalcMetrics(o);
            return o.autoAlignMetrics[METRIC_IL][0];
        }
        std::vector<double> zc = z, zBest = z;   // round start (trust box centre), best re-selected point
        double fBest = f;
        // inverse Hessian estimate, initially a scaled identity (first step of unit length)
        std::vector<double> Hi((size_t)n * n, 0.0);
        double gn = 0.0;
        for (double v : gz) gn += v * v;
        gn = std::sqrt(gn);
        for (int i = 0; i < n; i++) Hi[(size_t)i * n + i] = 1.0 / std::max(gn, 1e-12);
        // convergence in dB, after the plain search's termination rule (a sweep
        // gaining at most the tolerance ends a pass, digHolo.cpp:12416, 12872):
        // the goal's pass at the user's tolerance (a tenth of it for MDL, whose
        // objective bends where its extreme eigenvalues cross), the IL pass
        // before an MDL goal at the reference's loose first-pass tolerance
        // 0.1 + 10 tol (digHolo.cpp:12462)
        const double userTol = (double)c.autoAlignTol;
        const double tol = pass + 1 < passes ? std::max(1e-4, 0.1 + 10.0 * userTol)
                           : std::max(1e-4, metric == METRIC_MDL ? 0.1 * userTol : userTol);
        const int maxIter = 80, maxRounds = 8;
        int quiet = 0, round = 0;
        bool firstUpdate = true, restarted = false;
        double lastRoundEnd = f;   // objective at the end of the previous round (before re-selection)
        std::vector<double> d(n), s(n), y(n), Hy(n);
        for (int it = 0; it < maxIter; it++) {
            double slope = 0.0;
            for (int i = 0; i < n; i++) {
                double v = 0.0;
                for (int j = 0; j < n; j++) v -= Hi[(size_t)i * n + j] * gz[j];
                d[i] = v;
                slope += v * gz[i];
            }
            if (slope >= 0) {   // not a descent direction: restart from the gradient
                for (int i = 0; i < n; i++) {
                    for (int j = 0; j < n; j++) Hi[(size_t)i * n + j] = (i == j) ? 1.0 / std::max(gn, 1e-12) : 0.0;
                    d[i] = -gz[i] / std::max(gn, 1e-12);
                }
                slope = 0.0;
                for (int i = 0; i < n; i++) slope += d[i] * gz[i];
            }
            double t = 1.0, ft = 0.0;
            bool accepted = false;
            bool boxed = false;
            for (int ls = 0; ls < 6; ls++) {
                boxed = false;
                for (int i = 0; i < n; i++) {
                    zt[i] = z[i] + t * d[i];
                    if (isTilt[i] && std::fabs(zt[i] - zc[i]) > tiltTrust) {
                        zt[i] = zc[i] + (zt[i] > zc[i] ? tiltTrust : -tiltTrust);
                        boxed = true;
                    }
                }
                if (evalV(zt, ft)) return -FLT_MAX;
                if (ft <= f + 1e-4 * t * slope) {
                    if (evalG(gt)) return -FLT_MAX;
                    accepted = true;
                    break;
                }
                // minimiser of the quadratic through f, slope and ft, kept in [0.1 t, 0.5 t]
                const double tq = -slope * t * t / (2.0 * (ft - f - slope * t));
                t = std::min(0.5 * t, std::max(0.1 * t, tq));
            }
            if (!accepted) {
                // the quasi-Newton direction failed: once, restart from the
                // scaled gradient before giving up (the MDL objective bends
                // where its extreme eigenvalues cross)
                if (!restarted) {
                    restarted = true;
                    firstUpdate = true;
                    for (size_t i = 0; i < Hi.size(); i++) Hi[i] = 0.0;
                    for (int i = 0; i < n; i++) Hi[(size_t)i * n + i] = 1.0 / std::max(gn, 1e-12);
                    continue;
                }
                apply(z);
                break;
            }
            restarted = false;
            double sy = 0.0;
            for (int i = 0; i < n; i++) {
                s[i] = zt[i] - z[i];
                y[i] = gt[i] - gz[i];
                sy += s[i] * y[i];
            }
            const double df = f - ft;
            z = zt;
            gz = gt;
            f = ft;
            gn = 0.0;
            for (double v : gz) gn += v * v;
            gn = std::sqrt(gn);
            if (sy > 1e-12) {
                if (firstUpdate) {
                    // scale the initial estimate by s.y / y.y before the first update
                    double yy = 0.0;
                    for (int i = 0; i < n; i++) yy += y[i] * y[i];
                    for (size_t i = 0; i < Hi.size(); i++) Hi[i] = 0.0;
                    for (int i = 0; i < n; i++) Hi[(size_t)i * n + i] = sy / yy;
                    firstUpdate = false;
                }
                // BFGS update of the inverse Hessian
                double yHy = 0.0;
                for (int i = 0; i < n; i++) {
                    double v = 0.0;
                    for (int j = 0; j < n; j++) v += Hi[(size_t)i * n + j] * y[j];
                    Hy[i] = v;
                    yHy += y[i] * v;
                }
                const double rho = 1.0 / sy;
                for (int i = 0; i < n; i++)
                    for (int j = 0; j < n; j++)
                        Hi[(size_t)i * n + j] += (1.0 + yHy * rho) * rho * s[i] * s[j] - rho * (Hy[i] * s[j] + s[i] * Hy[j]);
            }
            // converged: a step below the tolerance and a predicted gain of the
            // next quasi-Newton step (g' H^-1 g / 2) below it too, or two small steps
            double decrement = 0.0;
            for (int i = 0; i < n; i++) {
                double v = 0.0;
                for (int j = 0; j < n; j++) v += Hi[(size_t)i * n + j] * gz[j];
                decrement += 0.5 * v * gz[i];
            }
            quiet = (df < tol) ? quiet + 1 : 0;
            if ((quiet >= 1 && decrement < tol) || quiet >= 2 || boxed) {
                // converged with these windows, or at the edge of the round's
                // tilt box: re-select the windows at the reached point, unless
                // the last re-selection and its round gained too little
                const double gain = lastRoundEnd - f;
                if (++round >= maxRounds || (round > 1 && gain < tol && !boxed)) break;
                lastRoundEnd = f;
                Config snap = c;
                snap.apertureSize = o.ifftSnap.apertureSize;
                // a selection that comes out as the held one re-evaluates nothing
                const bool same = sameSelection(o, o.ifftSnap, snap);
                o.ifftSnap = snap;
                if (!same && evalF(z, f, gz)) return -FLT_MAX;
                if (f < fBest) { fBest = f; zBest = z; }
                zc = z;
                quiet = 0;
            }
        }
        // the reached point with its windows re-selected, against the best
        // re-selected point of the pass
        {
            apply(z);
            Config snap = c;
            snap.apertureSize = o.ifftSnap.apertureSize;
            const bool same = sameSelection(o, o.ifftSnap, snap);
            o.ifftSnap = snap;
            double fz = f;
            if (!same && evalF(z, fz, gz)) return -FLT_MAX;
            if (fz > fBest) z = zBest;
        }
        apply(z);
    }
    // final pass and the metrics of the reached configuration, with the
    // Fourier window re-selected there and the FFT window still where the
    // search found it (the reference's search moves the FFT window only at
    // the next digHoloFFT either)
    {
        Config snap = c;
        snap.apertureSize = o.ifftSnap.apertureSize;
        o.ifftSnap = snap;
    }
    // the last evaluation already ran this configuration with these windows
    // (its coefficients are on the device) unless the search returned to an
    // earlier point
    const bool current = haveLast && memcmp(&lastCfg, &c, sizeof(Config)) == 0 && sameSelection(o, lastSnap, o.ifftSnap);
    if (!current) {
        if (objProcessForAlign(o)) return -FLT_MAX;
        o.alignEvaluations++;
    }
    objCalcMetrics(o);
    objCoefsToHost(o);
    return o.autoAlignMetrics[c.autoAlignGoalIdx][0];
}

}  // namespace dh
