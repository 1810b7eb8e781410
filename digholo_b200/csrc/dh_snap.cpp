// AutoAlign parameter estimate (digHoloAutoAlignSnap, digHolo.cpp:11517-11970)
// and the focus search it ends with (digHoloAutoFocus, digHolo.cpp:11181-11499),
// the start of AutoAlign modes FULL and ESTIMATE.  The host follows the
// reference's steps; every per-pixel stage runs in the kernels of dh_snap.cu:
//   1. beam centres reset to the middle of each polarisation's half of the
//      frame, tilts and defocus to zero (for the enabled parameters);
//   2. FFT windows of the whole half frame; R2C planes of every frame;
//   3. per polarisation, the tilt from the correlation of the batch-summed
//      Fourier intensity with the Fourier window (DCT-II, Gaussian filter,
//      DCT-III, maximum outside the DC disk); with AutoAlignFourierWindowRadius
//      the window radius shrinks to |tilt| / 3 (two passes then); the
//      Fourier-plane waist from the effective area inside the window;
//   4. the reconstructed fields of the whole half frame: beam centre from the
//      centre of mass and waist from the effective area of their summed
//      intensity, a defocus scale from the two waists;
//   5. the focus search over the tilt-removed fields.
// The reference runs stage 4 and 5 on the planes of stage 2 and the
// configuration of the moment, and so does this file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "dh_object.h"
#include "dh_snap.h"

namespace dh {

float fitToQuadratic(const float* x, const float* y, int n, float* B, const float* B0, float tol, float maxIter);

static const float PI_F = 3.14159265358979323846264338327950288f;
static const double PI_D = 3.14159265358979323846264338327950288;
static const float UNIT_ANGLE = PI_F / 180.0f;

namespace {

// AeffToMFD (digHolo.cpp:2887-2900)
float aeffToMfd(float aeff, int groups) {
    if (!groups) return 0.f;
    const float A = (float)(aeff / (15.1059697707643 * groups + 6.65360122093789));
    return 1.0f * (float)(2 * sqrtf(A / PI_F) / 0.223008930683135);
}

// FocusEstimate (digHolo.cpp:12017-12050)
float focusEstimate(float wCamera, float wFourier) {
    if (!(wCamera > 0 && wFourier > 0)) return 0.f;
    const float ratio = wFourier / wCamera;
    const float a = 0.25f, b = PI_F / 2;
    float r = 1.0f * 2 * (b * sqrtf((1 - a) / (ratio - a) - 1));
    if (!(r > 0)) r = 0.f;
    if (std::isnan(r)) r = 0.f;
    return r;
}

struct Tables {
    DhMixPlan plan;
    DevBuf tw;
};

int twiddles(Object& o, int N, Tables& t) {
    if (!dh_mix_plan(N, t.plan)) return fail(o, ERR_INVALIDDIMENSION, "AutoAlign estimate: a transform length has a prime factor above 64");
    std::vector<float> h(2 * (size_t)N);
    for (int k = 0; k < N; k++) {
        const double a = -2.0 * PI_D * (double)k / (double)N;
        h[2 * k] = (float)std::cos(a);
        h[2 * k + 1] = (float)std::sin(a);
    }
    DH_CUDA(o, t.tw.ensure(h.size() * sizeof(float)));
    DH_CUDA(o, cudaMemcpyAsync(t.tw.ptr, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, o.stream));
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    return ERR_SUCCESS;
}

// cos(pi m / (2 n)) for m < 4 n: the DCT kernels' table
int cosTable(Object& o, int n, DevBuf& d) {
    std::vector<double> h(4 * (size_t)n);
    for (int m = 0; m < 4 * n; m++) h[m] = std::cos(PI_D * (double)m / (2.0 * (double)n));
    DH_CUDA(o, d.ensure(h.size() * sizeof(double)));
    DH_CUDA(o, cudaMemcpy(d.ptr, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    return ERR_SUCCESS;
}

int upload(Object& o, DevBuf& d, const void* src, size_t bytes) {
    DH_CUDA(o, d.ensure(bytes));
    DH_CUDA(o, cudaMemcpy(d.ptr, src, bytes, cudaMemcpyHostToDevice));
    return ERR_SUCCESS;
}

// 2D transform of `units` planes of ny rows by nx columns, in place, or
// from `in` to `out`: rows, then columns; `sum` (optional) receives
// sum |.|^2 per polarisation and pixel instead of the column pass's output.
int fft2d(Object& o, const float2* in, float2* out, int units, int P, int nx, int ny, const Tables& tx,
          const Tables& ty, int inverse, const short* ref, float* sum) {
    DhSnapFftArgs a;
    memset(&a, 0, sizeof(a));
    a.in = in;
    a.out = out;
    a.unitStride = (size_t)nx * ny;
    a.units = units;
    a.vecs = ny;
    a.vecStride = nx;
    a.elemStride = 1;
    a.G = std::max(1, std::min(dh_snap_vectors_per_block(nx), ny));
    a.inverse = inverse;
    a.plan = tx.plan;
    a.tw = tx.tw.as<float2>();
    a.polCount = P;
    a.ref = ref;
    a.nx = nx;
    a.ny = ny;
    DH_CUDA(o, dh_launch_snap_fft(a, o.stream));
    DhSnapFftArgs b = a;
    b.in = out;
    b.vecs = nx;
    b.vecStride = 1;
    b.elemStride = nx;
    b.G = std::max(1, std::min(dh_snap_vectors_per_block(ny), nx));
    b.plan = ty.plan;
    b.tw = ty.tw.as<float2>();
    b.ref = nullptr;
    b.sum = sum;
    b.sumStride = (size_t)nx * ny;
    DH_CUDA(o, dh_launch_snap_fft(b, o.stream));
    return ERR_SUCCESS;
}

}  // namespace

// Runs the estimate on the handle's batch and leaves the estimated tilt,
// beam centre, waist, defocus (and, with AutoAlignFourierWindowRadius, the
// Fourier window radius) in o.cfg; steps[] receives the search step sizes
// the reference derives from them (tilt, centre, defocus, waist).
int objAutoAlignSnap(Object& o, float steps[4]) {
    Config& c = o.cfg;
    const int P = c.polCount;
    const int fw = c.frameWidth, fh = c.frameHeight;
    const float ps = c.pixelSize;
    int r = objInitDevice(o);
    if (r) return r;
    if (!o.frames) return fail(o, ERR_NULLPOINTER, "frame buffer not set");
    if (c.avgCount > 1) return fail(o, ERR_INVALIDARGUMENT, "AutoAlign estimate: frame averaging (avgCount > 1) is not supported");
    if (o.framesTransposed) return fail(o, ERR_INVALIDARGUMENT, "AutoAlign estimate: transposed frames are not supported");
    const int B = std::max(1, c.batchCount);
    const int units = B * P;
    const size_t es = o.framesU16 ? 2 : 4;

    // frames on the device (host batches are copied whole)
    const void* frames = o.frames;
    {
        cudaPointerAttributes pa;
        const bool dev = cudaPointerGetAttributes(&pa, o.frames) == cudaSuccess &&
                         (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
        cudaGetLastError();
        if (!dev) {
            const size_t bytes = (size_t)B * fw * fh * es;
            DH_CUDA(o, o.dAlignFrames.ensure(bytes));
            DH_CUDA(o, cudaMemcpy(o.dAlignFrames.ptr, o.frames, bytes, cudaMemcpyHostToDevice));
            frames = o.dAlignFrames.ptr;
        }
    }

    // 1. reset (digHolo.cpp:11525-11548)
    for (int p = 0; p < P; p++) {
        if (c.autoAlignCentre) {
            c.beamCentreX[p] = (float)((-(P - 1) * (fw / 4.0) + (p * fw / 2.0)) * c.pixelSize);
            c.beamCentreY[p] = 0;
        }
        if (c.autoAlignTilt) { c.zern[p][ZERN_TILTX] = 0; c.zern[p][ZERN_TILTY] = 0; }
        if (c.autoAlignDefocus) c.zern[p][ZERN_DEFOCUS] = 0;
    }
    // 2. the whole half frame as FFT window (digHolo.cpp:11553-11560)
    Config s = c;
    s.fftWindowSizeX = fw / P;
    s.fftWindowSizeY = fh;
    Geometry g;
    fftWindowGeometry(s, P, g);
    const int W = g.W, H = g.H, Nx = W / 2 + 1;
    Tables tW, tH;
    if ((r = twiddles(o, W, tW)) || (r = twiddles(o, H, tH))) return r;
    DevBuf& dPlane = o.dSnap[0];
    DH_CUDA(o, dPlane.ensure((size_t)units * H * Nx * sizeof(float2)));
    {
        DhSnapPlaneArgs a;
        memset(&a, 0, sizeof(a));
        a.frames = frames;
        a.u16 = o.framesU16;
        a.frameWidth = fw;
        a.frameStride = (long long)fw * fh;
        for (int p = 0; p < P; p++) { a.cx[p] = g.cx[p]; a.cy[p] = g.cy[p]; }
        a.W = W;
        a.H = H;
        a.polCount = P;
        a.units = units;
        a.G = std::max(1, std::min(dh_snap_vectors_per_block(W), H));
        a.planW = tW.plan;
        a.twW = tW.tw.as<float2>();
        a.plane = dPlane.as<float2>();
        DH_CUDA(o, dh_launch_snap_plane_rows(a, o.stream));
        DhSnapFftArgs b;
        memset(&b, 0, sizeof(b));
        b.in = b.out = dPlane.as<float2>();
        b.unitStride = (size_t)H * Nx;
        b.units = units;
        b.vecs = Nx;
        b.vecStride = 1;
        b.elemStride = Nx;
        b.G = std::max(1, std::min(dh_snap_vectors_per_block(H), Nx));
        b.plan = tH.plan;
        b.tw = tH.tw.as<float2>();
        b.polCount = P;
        DH_CUDA(o, dh_launch_snap_fft(b, o.stream));
    }
    DevBuf &dAx = o.dSnap[1], &dS = o.dSnap[2], &dS0 = o.dSnap[3], &dD = o.dSnap[4], &dCorr = o.dSnap[5],
           &dCosN = o.dSnap[6], &dCosH = o.dSnap[7], &dSmall = o.dSnap[8];
    {
        std::vector<float> ax(g.kx);
        ax.insert(ax.end(), g.ky.begin(), g.ky.end());
        if ((r = upload(o, dAx, ax.data(), ax.size() * sizeof(float)))) return r;
    }
    const float* dKx = dAx.as<float>();
    const float* dKy = dKx + W;
    const float k0 = 2 * PI_F / c.wavelengthCentre;
    auto batchSums = [&](bool both) -> int {
        const float R = 2 * k0 * sinf(c.apertureSize * UNIT_ANGLE);   // digHolo.cpp:6936-6939
        DH_CUDA(o, dS.ensure((size_t)P * H * Nx * sizeof(float)));
        DH_CUDA(o, dh_launch_snap_batchsum(dPlane.as<float2>(), B, P, H, Nx, dKx, dKy, R * R, dS.as<float>(), o.stream));
        if (both) {
            DH_CUDA(o, dS0.ensure((size_t)P * H * Nx * sizeof(float)));
            DH_CUDA(o, dh_launch_snap_batchsum(dPlane.as<float2>(), B, P, H, Nx, dKx, dKy, 0.f, dS0.as<float>(), o.stream));
        }
        return ERR_SUCCESS;
    };
    if ((r = batchSums(true))) return r;
    if ((r = cosTable(o, Nx, dCosN)) || (r = cosTable(o, H, dCosH))) return r;
    DH_CUDA(o, dD.ensure((size_t)H * Nx * sizeof(double)));
    DH_CUDA(o, dCorr.ensure((size_t)2 * H * Nx * sizeof(float)));
    DH_CUDA(o, dSmall.ensure(4096));
    const float dAk = std::fabs(g.kx[2] - g.kx[1]) * std::fabs(g.ky[2] - g.ky[1]);

    // 3. tilt and Fourier-plane waist (digHolo.cpp:11587-11788)
    float waistF[POLMAX] = {0.f, 0.f};
    const int passCount = 1 + (c.autoAlignFourierWindowRadius ? 1 : 0);
    for (int pass = 0; pass < passCount; pass++) {
        for (int p = 0; p < P; p++) {
            const float apRad = c.apertureSize * UNIT_ANGLE;
            const float aperturek = k0 * apRad;
            const float wx = (float)((1.0 * PI_F / aperturek) * std::sqrt(2.0));
            const float wy = (float)((2.0 * PI_F / aperturek) * std::sqrt(2.0));
            const float wx2 = (float)(-1.0 / (double)(wx * wx));
            const float wy2 = (float)(-1.0 / (double)(wy * wy));
            float* corr = dCorr.as<float>();
            float* corr2 = corr + (size_t)H * Nx;
            const float* Sp = dS.as<float>() + (size_t)p * H * Nx;
            DH_CUDA(o, dh_launch_snap_dct(Sp, nullptr, dD.as<double>(), nullptr, H, Nx, 1, 2, dCosN.as<double>(), o.stream));
            DH_CUDA(o, dh_launch_snap_dct(nullptr, dD.as<double>(), nullptr, corr, H, Nx, 0, 2, dCosH.as<double>(), o.stream));
            DH_CUDA(o, dh_launch_snap_filter(corr, H, Nx, wx2, wy2, ps, ps * ps, o.stream));
            DH_CUDA(o, dh_launch_snap_dct(corr, nullptr, dD.as<double>(), nullptr, H, Nx, 1, 3, dCosN.as<double>(), o.stream));
            DH_CUDA(o, dh_launch_snap_dct(nullptr, dD.as<double>(), nullptr, corr2, H, Nx, 0, 3, dCosH.as<double>(), o.stream));
            float ad = aperturek * 2;
            ad = ad * ad;
            int idx = -1;
            DH_CUDA(o, dh_launch_snap_argmax(corr2, 1, H, Nx, dKx, dKy, ad, 0, dSmall.as<int>(), o.stream));
            DH_CUDA(o, cudaMemcpyAsync(&idx, dSmall.ptr, sizeof(int), cudaMemcpyDeviceToHost, o.stream));
            DH_CUDA(o, cudaStreamSynchronize(o.stream));
            float tx = 0.f, ty = 0.f;
            if (idx >= 0) {
                const int j = idx / Nx, i = idx % Nx;
                tx = asinf(g.kx[i] / k0) / UNIT_ANGLE;
                ty = asinf(g.ky[j] / k0) / UNIT_ANGLE;
            }
            if (c.autoAlignFourierWindowRadius) {
                const float apMax = sqrtf(tx * tx + ty * ty) / 3.0f;   // FourierWindowRadiusRec
                if (apMax < c.apertureSize) {
                    c.apertureSize = apMax;
                    if ((r = batchSums(false))) return r;   // digHoloFFTAnalysis with the new radius
                }
            }
            if (c.autoAlignTilt) { c.zern[p][ZERN_TILTX] = tx; c.zern[p][ZERN_TILTY] = ty; }
            const float cxy[2] = {k0 * (c.zern[p][ZERN_TILTX] * UNIT_ANGLE), k0 * (c.zern[p][ZERN_TILTY] * UNIT_ANGLE)};
            const float wr = k0 * sinf(c.apertureSize * UNIT_ANGLE);
            float* dCxy = reinterpret_cast<float*>(dSmall.as<char>() + 64);
            double* dMom = reinterpret_cast<double*>(dSmall.as<char>() + 128);
            DH_CUDA(o, cudaMemcpyAsync(dCxy, cxy, sizeof(cxy), cudaMemcpyHostToDevice, o.stream));
            DH_CUDA(o, dh_launch_snap_moments(dS0.as<float>() + (size_t)p * H * Nx, 1, H, Nx, 0, dKx, dKy, 1, dCxy,
                                              wr * wr, dMom, o.stream));
            double mom[4];
            DH_CUDA(o, cudaMemcpyAsync(mom, dMom, sizeof(mom), cudaMemcpyDeviceToHost, o.stream));
            DH_CUDA(o, cudaStreamSynchronize(o.stream));
            const float aeff = (float)((double)dAk * mom[0] * mom[0] / mom[3]);
            const float wEst = aeffToMfd(aeff, c.maxMG);
            waistF[p] = (float)((1.0 / wEst) * PI_F);
        }
    }

    // 4. reconstructed fields of the whole half frame (digHolo.cpp:11791-11902)
    float maxFocus = 0.25f;
    float est[POLMAX] = {0.f, 0.f};
    bool valid = false;
    int attempts = 0;
    Geometry g2 = g;
    DevBuf &dField = o.dSnap[9], &dTmp = o.dSnap[10], &dAdj = o.dSnap[11], &dFS = o.dSnap[12], &dAxes = o.dSnap[13];
    Tables tx, ty;
    Config s2 = s;
    while ((!valid || attempts == 0) && attempts < 10) {
        valid = true;
        s2 = c;
        s2.fftWindowSizeX = s.fftWindowSizeX;
        s2.fftWindowSizeY = s.fftWindowSizeY;
        g2 = g;
        ifftWindowGeometry(s2, P, g2);
        const int nx = g2.nx, ny = g2.ny;
        if ((r = twiddles(o, nx, tx)) || (r = twiddles(o, ny, ty))) return r;
        std::vector<float> adj;
        windowFactors(s2, s2, g2, P, adj);
        if ((r = upload(o, dAdj, adj.data(), adj.size() * sizeof(float)))) return r;
        DH_CUDA(o, dField.ensure((size_t)units * nx * ny * sizeof(float2)));
        DhSnapPlaceArgs pa;
        memset(&pa, 0, sizeof(pa));
        pa.plane = dPlane.as<float2>();
        pa.adj = dAdj.as<float2>();
        pa.field = dField.as<float2>();
        pa.W = W; pa.H = H; pa.w = g2.w; pa.h = g2.h; pa.nx = nx; pa.ny = ny;
        pa.lowres = s2.resolutionIdx != 0;
        pa.polCount = P;
        pa.units = units;
        for (int p = 0; p < P; p++) { pa.sx0[p] = g2.SX[p] - W / 2; pa.SY[p] = g2.SY[p]; }
        DH_CUDA(o, dh_launch_snap_place(pa, o.stream));
        if ((r = fft2d(o, dField.as<float2>(), dField.as<float2>(), units, P, nx, ny, tx, ty, 1, nullptr, nullptr)))
            return r;
        DH_CUDA(o, dFS.ensure((size_t)P * nx * ny * sizeof(float)));
        DH_CUDA(o, dh_launch_snap_field_sum(dField.as<float2>(), B, P, (size_t)nx * ny, (float)(1.0 / ((double)nx * ny)),
                                            dFS.as<float>(), o.stream));
        std::vector<float> axes(g2.x);
        axes.insert(axes.end(), g2.y.begin(), g2.y.end());
        if ((r = upload(o, dAxes, axes.data(), axes.size() * sizeof(float)))) return r;
        double* dMom = reinterpret_cast<double*>(dSmall.as<char>() + 128);
        DH_CUDA(o, dh_launch_snap_moments(dFS.as<float>(), P, ny, nx, (size_t)nx * ny, dAxes.as<float>(),
                                          dAxes.as<float>() + nx, 0, nullptr, 0.f, dMom, o.stream));
        double mom[POLMAX * 4];
        DH_CUDA(o, cudaMemcpyAsync(mom, dMom, sizeof(double) * 4 * P, cudaMemcpyDeviceToHost, o.stream));
        DH_CUDA(o, cudaStreamSynchronize(o.stream));
        const float dA = std::fabs(g2.x[2] - g2.x[1]) * std::fabs(g2.y[2] - g2.y[1]);
        for (int p = 0; p < P; p++) {
            const float polOffsetX = (float)(((2 * p - 1) * c.pixelSize * fw / 4.0) * (P - 1));
            const double* m = mom + 4 * p;
            const float comx = (float)(m[1] / m[0]) + polOffsetX;
            const float comy = (float)(m[2] / m[0]);
            const float aeff = (float)((double)dA * m[0] * m[0] / m[3]);
            const float wEst = (float)(aeffToMfd(aeff, c.maxMG) * 0.5);
            est[p] = focusEstimate(wEst, waistF[p]);
            if (std::isnan(comx) || std::isnan(comy) || std::isnan(aeff)) {
                valid = false;
                c.apertureSize *= 0.9f;
            }
            if (valid) {
                if (c.autoAlignCentre) { c.beamCentreX[p] = comx; c.beamCentreY[p] = comy; }
                if (c.autoAlignBasisWaist) c.waist[p] = wEst;
                if (c.autoAlignDefocus) c.zern[p][ZERN_DEFOCUS] = 0;
                if (std::fabs(est[p]) > maxFocus) maxFocus = std::fabs(est[p]);
            }
            attempts++;
        }
    }

    // 5. focus search (digHoloAutoFocus, digHolo.cpp:11181-11499) on the
    // fields of the last pass above; the reference wave follows the
    // configuration as it is now, with the trial defocus
    if (c.autoAlignDefocus) {
        const int nx = g2.nx, ny = g2.ny;
        const float dAf = std::fabs(g.kx[2] - g.kx[1]) * std::fabs(g.ky[2] - g.ky[1]);
        DH_CUDA(o, dTmp.ensure((size_t)units * nx * ny * sizeof(float2)));
        DevBuf& dRef = o.dSnap[14];
        const int stepCount = 25, stepFitCount = 5;
        float scale[POLMAX], scale0[POLMAX];
        float defoc[POLMAX][stepCount + 3] = {}, aeffs[POLMAX][stepCount + 3] = {};
        float bestAeff[POLMAX] = {FLT_MAX, FLT_MAX}, best[POLMAX] = {0.f, 0.f};
        int converged[POLMAX] = {0, 0};
        float B0[POLMAX][3] = {}, Bq[POLMAX][3] = {};
        for (int p = 0; p < P; p++) {
            scale[p] = std::max(est[p], 1.0f);
            scale0[p] = scale[p];
        }
        for (int st = 0; st < stepCount; st += 2)
            for (int p = 0; p < P; p++) {
                defoc[p][st] = scale0[p];
                defoc[p][st + 1] = -scale0[p];
                scale0[p] += scale[p] * 0.25f;
            }
        bool total = false;
        for (int st = 0; st < stepCount && !total; st++) {
            total = true;
            Config t = s2;
            for (int p = 0; p < P; p++) {
                t.beamCentreX[p] = c.beamCentreX[p];
                t.beamCentreY[p] = c.beamCentreY[p];
                t.zern[p][ZERN_DEFOCUS] = defoc[p][st];
            }
            std::vector<short> ref;
            referenceWave(t, P, g2, ref);
            if ((r = upload(o, dRef, ref.data(), ref.size() * sizeof(short)))) return r;
            DH_CUDA(o, dFS.ensure((size_t)P * nx * ny * sizeof(float)));
            DH_CUDA(o, cudaMemsetAsync(dFS.ptr, 0, (size_t)P * nx * ny * sizeof(float), o.stream));
            if ((r = fft2d(o, dField.as<float2>(), dTmp.as<float2>(), units, P, nx, ny, tx, ty, 1, dRef.as<short>(),
                           dFS.as<float>())))
                return r;
            double* dMom = reinterpret_cast<double*>(dSmall.as<char>() + 128);
            DH_CUDA(o, dh_launch_snap_moments(dFS.as<float>(), P, ny, nx, (size_t)nx * ny, dAxes.as<float>(),
                                              dAxes.as<float>() + nx, 0, nullptr, 0.f, dMom, o.stream));
            double mom[POLMAX * 4];
            DH_CUDA(o, cudaMemcpyAsync(mom, dMom, sizeof(double) * 4 * P, cudaMemcpyDeviceToHost, o.stream));
            DH_CUDA(o, cudaStreamSynchronize(o.stream));
            for (int p = 0; p < P; p++) {
                const double v2 = mom[4 * p], v4 = mom[4 * p + 3];
                const float a = (float)((double)dAf * v2 * v2 / v4);
                aeffs[p][st] = a;
                if (a < bestAeff[p]) { bestAeff[p] = a; best[p] = defoc[p][st]; }
                if (st == 1) {
                    float stepScale, base;
                    if (aeffs[p][1] < aeffs[p][0]) { stepScale = defoc[p][1] - defoc[p][0]; base = defoc[p][1]; }
                    else { stepScale = defoc[p][0] - defoc[p][1]; base = defoc[p][0]; }
                    int idx = 1;
                    for (int i = st + 1; i < stepCount; i += 2) {
                        defoc[p][i] = base + idx * 0.25f * stepScale;
                        defoc[p][i + 1] = base - idx * 0.25f * stepScale;
                        idx++;
                    }
                }
                if (st >= stepFitCount - 1) {
                    if (st == stepFitCount - 1) {
                        B0[p][0] = 1e7f;
                        B0[p][1] = 1e7f;
                        B0[p][2] = 0;
                        for (int i = 0; i < st; i++) B0[p][2] += aeffs[p][i] / (st + 1);
                    }
                    float xs[stepCount + 3], ys[stepCount + 3];
                    for (int i = 0; i <= st; i++) { xs[i] = defoc[p][i]; ys[i] = aeffs[p][i]; }
                    // sortIt (digHolo.cpp:11161-11179): ascending effective area
                    for (int a2 = 0; a2 <= st; a2++)
                        for (int b2 = 1; b2 <= st; b2++)
                            if (ys[b2] < ys[b2 - 1]) { std::swap(ys[b2], ys[b2 - 1]); std::swap(xs[b2], xs[b2 - 1]); }
                    const float mx = fitToQuadratic(xs, ys, stepFitCount - 1, Bq[p], B0[p], 1e-6f, 1000);
                    memcpy(B0[p], Bq[p], sizeof(B0[p]));
                    if (st + 1 < stepCount - 1 && !std::isnan(mx)) defoc[p][st + 1] = mx;
                    if (std::fabs(mx - best[p]) < 0.01f) converged[p] = 1;
                }
                total = total && converged[p];
            }
        }
        for (int p = 0; p < P; p++) {
            c.zern[p][ZERN_DEFOCUS] = best[p];
            if (std::fabs(best[p]) > maxFocus) maxFocus = std::fabs(best[p]);
        }
    }
    // step sizes of the search that follows (digHolo.cpp:11955-11960)
    steps[0] = c.apertureSize * 0.1f;
    steps[1] = c.waist[0] * 0.1f;
    steps[2] = 0.1f * maxFocus;
    steps[3] = c.waist[0] * 0.1f;
    o.preparedValid = 0;
    return ERR_SUCCESS;
}

// AeffToMFD for the frame simulator's default beam waist.
float aeffToMfdPublic(float aeff, int groups) { return aeffToMfd(aeff, groups); }

}  // namespace dh
