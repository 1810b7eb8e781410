// Frame simulator: digHoloFrameSimulatorCreate / CreateSimple / Destroy
// (digHolo.h:2026-2056, digHolo.cpp:15686-16760) with the frames computed on
// the GPU (dh_sim.cu), and digHoloB200FrameSimulatorDevice, which leaves the
// frames in device memory.
//
// Parameters and their defaults follow frameSimulatorCreate
// (digHolo.cpp:15930-16330): frame sides floored to multiples of 16; pixel
// size 20 um; at most two polarisations, side by side; camera levels in
// [2, 65536] (else 65536); wavelength 1565 nm; reference tilt (tiltMax,
// -tiltMax) with tiltMax the largest tilt the widest window supports; no
// defocus, plane-wave reference centred on its region; beam waist from the
// effective area of a circle of a quarter of the region's smaller side;
// one-hot coefficients (frame f excites mode f in every polarisation); mode
// groups enough for one mode per frame when none are given.
//
// The reference's region axes are transposed against its frame layout
// (digHolo.cpp:16371-16385 with generateModeSeparable's transpose): its "x"
// axis (beam centre x, reference tilt x, the HG modes of index n) runs along
// the frame's rows, its "y" axis along the columns of a polarisation region.
// That convention is kept.  Deviations, on purpose:
//  - with no group count given and a frame count that is not a triangular
//    number, the reference fills its default coefficients with one mode
//    count and reads them with another (digHolo.cpp:16012-16027 against
//    16318-16343), so later frames read memory it never wrote; here the
//    one-hot coefficients use the final mode count;
//  - the reference builds one reference wave per wavelength from the mean
//    wavenumber (digHolo.cpp:16431-16482), i.e. identical waves; here the
//    wave is built once, the same values;
//  - refAmplitude is accepted and returned but, as in the reference, not
//    applied.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "dh_host.h"
#include "dh_object.h"
#include "dh_params.h"
#include "dh_sim.h"
#include "dh_snap.h"

cudaError_t dh_launch_basis_jobs(const DhBasisParams* ps, int n, cudaStream_t s);

namespace dh {
float aeffToMfdPublic(float aeff, int groups);
}

namespace {

const float PI_F = 3.14159265358979323846264338327950288f;   // digHolo.cpp:89
constexpr int POLMAX = 2;
constexpr int QUANTA = 16;
const double WMAXRATIO = 0.32037724101704079249230971981887705624103546142578125;
const float UNIT_ANGLE_F = PI_F / 180.0f;

struct SimSpec {
    int frames = 0, W = 0, H = 0, P = 1, G = 0, M = 0, levels = 65536, fill = 0;
    float ps = 20e-6f;
    float tiltX[POLMAX], tiltY[POLMAX], defocus[POLMAX], refWaist[POLMAX], refCx[POLMAX], refCy[POLMAX];
    float refAmp[POLMAX][2];
    float waist[POLMAX], cx[POLMAX], cy[POLMAX];
    std::vector<float> coefs;        // [frame][pol][mode] re, im
    std::vector<float> wavelengths;
    float k0 = 0.f;
    float offsetX[POLMAX];
};

// Mode count of the smallest group count whose modes reach frameCount, with
// the reference's rule for the group count when none is given
// (digHolo.cpp:16004-16033).
void groupsFor(int frameCount, int& G, int& M) {
    if (G <= 0) {
        int m = 0, g = 1;
        while (m < frameCount) { m += g; g++; }
        G = (m == frameCount) ? g - 1 : g;
    }
    M = G * (G + 1) / 2;
}

// frameSimulatorCreate's parameter resolution.  Null pointers take defaults.
int resolve(int frameCount, int& W, int& H, float& ps, int& P, const float* tiltX, const float* tiltY,
            const float* defocus, const float* refWaist, const float* refCx, const float* refCy, const float* refAmp,
            int& G, const float* waist, const float* coefs, const float* cx, const float* cy, int& levels, int fill,
            const float* wavelengths, int& wavelengthCount, SimSpec& s) {
    if (frameCount <= 0 || W <= 0 || H <= 0 || P <= 0) return dh::ERR_INVALIDARGUMENT;
    if (levels < 2 || levels > 65536) levels = 65536;
    W = QUANTA * (W / QUANTA);
    H = QUANTA * (H / QUANTA);
    if (ps <= 0) ps = 20e-6f;
    if (P > POLMAX) P = POLMAX;
    if (W <= 0 || H <= 0) return dh::ERR_INVALIDDIMENSION;
    groupsFor(frameCount, G, s.M);
    if (wavelengthCount <= 0 || !wavelengths) wavelengthCount = 1;
    s.frames = frameCount;
    s.W = W;
    s.H = H;
    s.ps = ps;
    s.P = P;
    s.G = G;
    s.levels = levels;
    s.fill = fill;
    const int width = H, height = W / P;   // the reference's region axes (rows, columns)
    for (int p = 0; p < P; p++)
        s.offsetX[p] = (float)((ps * (W / P) / 2.0) * (P * p - 1 * (P - 1)));
    s.wavelengths.assign(wavelengthCount, 1565e-9f);
    if (wavelengths) s.wavelengths.assign(wavelengths, wavelengths + wavelengthCount);
    float k0 = 0;
    for (int i = 0; i < wavelengthCount; i++) k0 += (2 * PI_F) / s.wavelengths[i];
    k0 = k0 / wavelengthCount;
    s.k0 = k0;
    const float lambda0 = 2 * PI_F / k0;
    const float wmax = lambda0 / (2 * ps);
    const float tiltMax = (float)(wmax * (1 - WMAXRATIO) / UNIT_ANGLE_F);
    for (int p = 0; p < P; p++) {
        s.tiltX[p] = tiltX ? tiltX[p] : tiltMax;
        s.tiltY[p] = tiltY ? tiltY[p] : -tiltMax;
        s.defocus[p] = defocus ? defocus[p] : 0.f;
        s.refCx[p] = refCx ? refCx[p] : s.offsetX[p];
        s.refCy[p] = refCy ? refCy[p] : 0.f;
        s.refWaist[p] = refWaist ? refWaist[p] : 0.f;
        s.refAmp[p][0] = refAmp ? refAmp[2 * p] : 1.f;
        s.refAmp[p][1] = refAmp ? refAmp[2 * p + 1] : 0.f;
        s.cx[p] = cx ? cx[p] : s.offsetX[p];
        s.cy[p] = cy ? cy[p] : 0.f;
    }
    if (waist) {
        for (int p = 0; p < P; p++) s.waist[p] = waist[p];
    } else {
        const int minDim = width < height ? width : height;
        const float r = (float)(0.25 * minDim * ps);
        const float aeff = PI_F * r * r;
        const float w = dh::aeffToMfdPublic(aeff, G) * 0.5f;
        for (int p = 0; p < P; p++) s.waist[p] = w;
    }
    const size_t n = (size_t)frameCount * P * s.M * 2;
    if (coefs) {
        s.coefs.assign(coefs, coefs + n);
    } else {
        s.coefs.assign(n, 0.f);
        for (int f = 0; f < frameCount; f++)
            for (int p = 0; p < P; p++)
                if (f < s.M) s.coefs[(((size_t)f * P + p) * s.M + f) * 2] = 1.f;
    }
    return dh::ERR_SUCCESS;
}

struct Dev {
    void* p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

#define SIM_CUDA(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { cudaGetLastError(); return dh::ERR_ERROR; } } while (0)

// The reference wave factor along one region axis (digHolo.cpp:16431-16482).
void refAxis(float kr, float kfocus, float w, float A0, const std::vector<float>& axis, float* out) {
    const float w2 = w * w;
    for (size_t i = 0; i < axis.size(); i++) {
        const float r = axis[i];
        const float r2 = r * r;
        const float arg = kr * r + kfocus * r2;
        const float A = w2 > 0 ? A0 * expf(-r2 / w2) : A0;
        out[2 * i] = A * cosf(arg);
        out[2 * i + 1] = A * sinf(arg);
    }
}

// The frames of `s` into device memory: float32 intensities (quantised,
// as the reference returns them) into d32 and, when d16 is given, uint16.
int simulate(const SimSpec& s, float* d32, unsigned short* d16, cudaStream_t st) {
    const int P = s.P, G = s.G, M = s.M;
    const int rows = s.H, cols = s.W / P;
    // region axes: rows (the reference's x) and columns (its y), per polarisation
    std::vector<float> axRow((size_t)P * rows), axCol((size_t)P * cols);
    std::vector<float> axRowRef((size_t)P * rows), axColRef((size_t)P * cols);
    for (int p = 0; p < P; p++) {
        const float xs = s.offsetX[p] - s.cx[p], ys = -s.cy[p];
        const float xr = s.offsetX[p] - s.refCx[p], yr = -s.refCy[p];
        for (int i = 0; i < rows; i++) {
            axRow[(size_t)p * rows + i] = s.ps * (i - rows / 2) + xs;
            axRowRef[(size_t)p * rows + i] = s.ps * (i - rows / 2) + xr;
        }
        for (int i = 0; i < cols; i++) {
            axCol[(size_t)p * cols + i] = s.ps * (i - cols / 2) + ys;
            axColRef[(size_t)p * cols + i] = s.ps * (i - cols / 2) + yr;
        }
    }
    // reference wave factors
    std::vector<float> refRow((size_t)P * rows * 2), refCol((size_t)P * cols * 2);
    for (int p = 0; p < P; p++) {
        const float kx = s.k0 * sinf(s.tiltX[p] * UNIT_ANGLE_F);
        const float ky = s.k0 * sinf(s.tiltY[p] * UNIT_ANGLE_F);
        const float kfocus = s.k0 * (0.5f * s.defocus[p]);
        std::vector<float> a(axRowRef.begin() + (size_t)p * rows, axRowRef.begin() + (size_t)(p + 1) * rows);
        refAxis(kx, kfocus, s.refWaist[p], sqrtf(1.0f / rows), a, &refRow[(size_t)p * rows * 2]);
        std::vector<float> b(axColRef.begin() + (size_t)p * cols, axColRef.begin() + (size_t)(p + 1) * cols);
        refAxis(ky, kfocus, s.refWaist[p], sqrtf(1.0f / cols), b, &refCol[(size_t)p * cols * 2]);
    }
    Dev dAxRow, dAxCol, dHgRow, dHgCol, dScale, dRefRow, dRefCol, dMax;
    SIM_CUDA(dAxRow.alloc(axRow.size() * 4));
    SIM_CUDA(dAxCol.alloc(axCol.size() * 4));
    SIM_CUDA(dHgRow.alloc((size_t)P * G * rows * 2));
    SIM_CUDA(dHgCol.alloc((size_t)P * G * cols * 2));
    SIM_CUDA(dScale.alloc((size_t)2 * P * G * 4));
    SIM_CUDA(dRefRow.alloc(refRow.size() * 4));
    SIM_CUDA(dRefCol.alloc(refCol.size() * 4));
    SIM_CUDA(dMax.alloc(4));
    SIM_CUDA(cudaMemcpyAsync(dAxRow.p, axRow.data(), axRow.size() * 4, cudaMemcpyHostToDevice, st));
    SIM_CUDA(cudaMemcpyAsync(dAxCol.p, axCol.data(), axCol.size() * 4, cudaMemcpyHostToDevice, st));
    SIM_CUDA(cudaMemcpyAsync(dRefRow.p, refRow.data(), refRow.size() * 4, cudaMemcpyHostToDevice, st));
    SIM_CUDA(cudaMemcpyAsync(dRefCol.p, refCol.data(), refCol.size() * 4, cudaMemcpyHostToDevice, st));
    SIM_CUDA(cudaMemsetAsync(dMax.p, 0, 4, st));
    // HG modes of every polarisation along both axes (HGbasisXY1D, FP64 recurrence)
    std::vector<DhBasisParams> jobs;
    for (int p = 0; p < P; p++) {
        DhBasisParams b;
        memset(&b, 0, sizeof(b));
        b.modes = G;
        b.modes16 = G;
        b.w0 = (double)s.waist[p];
        b.axis = dAxRow.as<float>() + (size_t)p * rows;
        b.count = rows;
        b.out16 = dHgRow.as<short>() + (size_t)p * G * rows;
        b.scale = dScale.as<float>() + (size_t)(0 * P + p) * G;
        jobs.push_back(b);
        b.axis = dAxCol.as<float>() + (size_t)p * cols;
        b.count = cols;
        b.out16 = dHgCol.as<short>() + (size_t)p * G * cols;
        b.scale = dScale.as<float>() + (size_t)(1 * P + p) * G;
        jobs.push_back(b);
    }
    SIM_CUDA(dh_launch_basis_jobs(jobs.data(), (int)jobs.size(), st));
    std::vector<float> scale((size_t)2 * P * G);
    SIM_CUDA(cudaMemcpyAsync(scale.data(), dScale.p, scale.size() * 4, cudaMemcpyDeviceToHost, st));
    SIM_CUDA(cudaStreamSynchronize(st));
    // the terms of every (frame, pol): modes with a nonzero coefficient, the
    // first and the last (generateModeSeparable's rule), in mode order
    std::vector<int> mIdx(M), nIdx(M);
    for (int g = 0, k = 0; g < G; g++)
        for (int q = 0; q <= g; q++, k++) { mIdx[k] = g - q; nIdx[k] = q; }
    std::vector<DhSimMode> terms;
    std::vector<int> offs((size_t)s.frames * P + 1, 0);
    int maxTerms = 1;
    for (int f = 0; f < s.frames; f++) {
        for (int p = 0; p < P; p++) {
            const size_t u = (size_t)f * P + p;
            offs[u] = (int)terms.size();
            const float* sc = &scale[(size_t)(0 * P + p) * G];   // rows (index n)
            const float* ss = &scale[(size_t)(1 * P + p) * G];   // columns (index m)
            for (int k = 0; k < M; k++) {
                const double xScale = ss[mIdx[k]], yScale = sc[nIdx[k]];
                const float* c = &s.coefs[(u * M + k) * 2];
                const float cR = (float)(xScale * yScale * c[0]);
                const float cI = (float)(xScale * yScale * c[1]);
                const float pw = cR * cR + cI * cI;
                if (pw > 0 || k == 0 || k == M - 1) terms.push_back({cR, cI, mIdx[k], nIdx[k]});
            }
            maxTerms = std::max(maxTerms, (int)terms.size() - offs[u]);
        }
    }
    offs[(size_t)s.frames * P] = (int)terms.size();
    Dev dTerms, dOffs;
    SIM_CUDA(dTerms.alloc(terms.size() * sizeof(DhSimMode)));
    SIM_CUDA(dOffs.alloc(offs.size() * sizeof(int)));
    SIM_CUDA(cudaMemcpyAsync(dTerms.p, terms.data(), terms.size() * sizeof(DhSimMode), cudaMemcpyHostToDevice, st));
    SIM_CUDA(cudaMemcpyAsync(dOffs.p, offs.data(), offs.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    DhSimFieldArgs fa;
    fa.modes = dTerms.as<DhSimMode>();
    fa.modeOffset = dOffs.as<int>();
    fa.hgCol = dHgCol.as<short>();
    fa.hgRow = dHgRow.as<short>();
    fa.refCol = dRefCol.as<float2>();
    fa.refRow = dRefRow.as<float2>();
    fa.out = d32;
    fa.maxBits = dMax.as<unsigned>();
    fa.frames = s.frames;
    fa.polCount = P;
    fa.rows = rows;
    fa.cols = cols;
    fa.frameWidth = s.W;
    fa.G = G;
    SIM_CUDA(dh_launch_sim_field(fa, maxTerms, st));
    if (s.fill) {
        // pixel fill factor: R2C of the whole frame, times sinc(kx ps/2)
        // sinc(ky ps/2) / (W H), C2R (digHolo.cpp:16508-16580, 15778-15830)
        const int W = s.W, H = s.H, Nx = W / 2 + 1;
        DhMixPlan planW, planH;
        if (!dh_mix_plan(W, planW) || !dh_mix_plan(H, planH)) return dh::ERR_INVALIDDIMENSION;
        const int Gw = dh_snap_vectors_per_block(W), Gh = dh_snap_vectors_per_block(H);
        if (Gw < 1 || Gh < 1) return dh::ERR_INVALIDDIMENSION;
        const double piD = 3.14159265358979323846;
        const float period = (float)(2.0 * s.ps);
        const float kfx = (float)(2 * (2.0 * piD / period) / W);
        const float kfy = (float)(2 * (2.0 * piD / period) / H);
        std::vector<float> sx(Nx), sy(H);
        for (int i = 0; i < Nx; i++) {
            const float k = kfx * (float)(i <= W / 2 ? i : i - W);
            const float a = k * 0.5f * s.ps;
            sx[i] = k != 0.f ? sinf(a) / a : 1.f;
        }
        for (int i = 0; i < H; i++) {
            const float k = kfy * (float)(i <= H / 2 ? i : i - H);
            const float a = k * 0.5f * s.ps;
            sy[i] = k != 0.f ? sinf(a) / a : 1.f;
        }
        std::vector<float> twW((size_t)W * 2), twH((size_t)H * 2);
        for (int k = 0; k < W; k++) {
            twW[2 * k] = (float)cos(-2.0 * piD * k / W);
            twW[2 * k + 1] = (float)sin(-2.0 * piD * k / W);
        }
        for (int k = 0; k < H; k++) {
            twH[2 * k] = (float)cos(-2.0 * piD * k / H);
            twH[2 * k + 1] = (float)sin(-2.0 * piD * k / H);
        }
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)s.frames, ((size_t)1 << 30) / ((size_t)H * W * 8 * 2)));
        Dev dHalf, dFull, dSx, dSy, dTwW, dTwH;
        SIM_CUDA(dHalf.alloc((size_t)chunk * H * Nx * 8));
        SIM_CUDA(dFull.alloc((size_t)chunk * H * W * 8));
        SIM_CUDA(dSx.alloc(sx.size() * 4));
        SIM_CUDA(dSy.alloc(sy.size() * 4));
        SIM_CUDA(dTwW.alloc(twW.size() * 4));
        SIM_CUDA(dTwH.alloc(twH.size() * 4));
        SIM_CUDA(cudaMemcpyAsync(dSx.p, sx.data(), sx.size() * 4, cudaMemcpyHostToDevice, st));
        SIM_CUDA(cudaMemcpyAsync(dSy.p, sy.data(), sy.size() * 4, cudaMemcpyHostToDevice, st));
        SIM_CUDA(cudaMemcpyAsync(dTwW.p, twW.data(), twW.size() * 4, cudaMemcpyHostToDevice, st));
        SIM_CUDA(cudaMemcpyAsync(dTwH.p, twH.data(), twH.size() * 4, cudaMemcpyHostToDevice, st));
        const float norm = 1.0f / (W * H);
        for (int f0 = 0; f0 < s.frames; f0 += chunk) {
            const int n = std::min(chunk, s.frames - f0);
            float* fr = d32 + (size_t)f0 * H * W;
            DhSnapPlaneArgs pa;
            memset(&pa, 0, sizeof(pa));
            pa.frames = fr;
            pa.u16 = 0;
            pa.frameWidth = W;
            pa.frameStride = (long long)W * H;
            pa.W = W;
            pa.H = H;
            pa.polCount = 1;
            pa.units = n;
            pa.G = Gw;
            pa.planW = planW;
            pa.twW = dTwW.as<float2>();
            pa.plane = dHalf.as<float2>();
            SIM_CUDA(dh_launch_snap_plane_rows(pa, st));
            DhSnapFftArgs fc;
            memset(&fc, 0, sizeof(fc));
            fc.in = dHalf.as<float2>();
            fc.out = dHalf.as<float2>();
            fc.unitStride = (size_t)H * Nx;
            fc.units = n;
            fc.vecs = Nx;
            fc.vecStride = 1;
            fc.elemStride = Nx;
            fc.G = Gh;
            fc.inverse = 0;
            fc.plan = planH;
            fc.tw = dTwH.as<float2>();
            fc.polCount = 1;
            SIM_CUDA(dh_launch_snap_fft(fc, st));
            SIM_CUDA(dh_launch_sim_sinc(dHalf.as<float2>(), n, H, Nx, dSx.as<float>(), dSy.as<float>(), norm, st));
            fc.inverse = 1;
            SIM_CUDA(dh_launch_snap_fft(fc, st));
            SIM_CUDA(dh_launch_sim_extend(dHalf.as<float2>(), dFull.as<float2>(), n, H, W, st));
            DhSnapFftArgs fr2 = fc;
            fr2.in = dFull.as<float2>();
            fr2.out = dFull.as<float2>();
            fr2.unitStride = (size_t)H * W;
            fr2.vecs = H;
            fr2.vecStride = W;
            fr2.elemStride = 1;
            fr2.G = Gw;
            fr2.plan = planW;
            fr2.tw = dTwW.as<float2>();
            fr2.inverse = 1;
            SIM_CUDA(dh_launch_snap_fft(fr2, st));
            SIM_CUDA(dh_launch_sim_real(dFull.as<float2>(), fr, (size_t)n * H * W, st));
        }
        SIM_CUDA(cudaStreamSynchronize(st));
    }
    SIM_CUDA(dh_launch_sim_quant(d32, d16, (size_t)s.frames * s.H * s.W, dMax.as<unsigned>(), s.levels, st));
    SIM_CUDA(cudaStreamSynchronize(st));
    return dh::ERR_SUCCESS;
}

int runOnDevice(const SimSpec& s, float* d32, unsigned short* d16) {
    int dev = 0, count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return dh::ERR_ERROR;
    }
    cudaGetDevice(&dev);
    cudaStream_t st;
    SIM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const int r = simulate(s, d32, d16, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return r;
}

}  // namespace

extern "C" {

// digHolo.h:2026.  Host memory: [float32 frames][uint16 frames][parameters],
// one allocation released by digHoloFrameSimulatorDestroy.
float* digHoloFrameSimulatorCreate(int frameCount, int* frameWidth, int* frameHeight, float* pixelSize, int* polCount,
                                   float** refTiltX, float** refTiltY, float** refDefocus, float** refWaist,
                                   float** refBeamCentreX, float** refBeamCentreY, float** refAmplitude,
                                   int* beamGroupCount, float** beamWaist, float** beamCoefs, float** beamCentreX,
                                   float** beamCentreY, int* cameraPixelLevelCount, int fillFactorCorrection,
                                   float** wavelengths, int* wavelengthCount, int wavelengthOrdering, int printToConsole,
                                   unsigned short** pixelBuffer16, const char* fname) {
    (void)wavelengthOrdering;
    if (!frameWidth || !frameHeight || !pixelSize || !polCount || !refTiltX || !refTiltY || !refDefocus || !refWaist ||
        !refBeamCentreX || !refBeamCentreY || !refAmplitude || !beamGroupCount || !beamWaist || !beamCoefs ||
        !beamCentreX || !beamCentreY || !cameraPixelLevelCount || !wavelengths || !wavelengthCount || !pixelBuffer16)
        return nullptr;
    SimSpec s;
    if (resolve(frameCount, *frameWidth, *frameHeight, *pixelSize, *polCount, *refTiltX, *refTiltY, *refDefocus,
                *refWaist, *refBeamCentreX, *refBeamCentreY, *refAmplitude, *beamGroupCount, *beamWaist, *beamCoefs,
                *beamCentreX, *beamCentreY, *cameraPixelLevelCount, fillFactorCorrection, *wavelengths,
                *wavelengthCount, s) != dh::ERR_SUCCESS)
        return nullptr;
    const int P = s.P, M = s.M, L = (int)s.wavelengths.size();
    const size_t n = (size_t)s.frames * s.H * s.W;
    const size_t params = (size_t)P * 6 + (size_t)P * 2 + (size_t)P * 3 + (size_t)s.frames * P * M * 2 + L;
    float* block = static_cast<float*>(malloc((n + (n + 1) / 2 + 2 + params) * sizeof(float)));
    if (!block) return nullptr;
    unsigned short* b16 = reinterpret_cast<unsigned short*>(block + n);
    float* prm = reinterpret_cast<float*>(b16 + n + ((n & 1) ? 1 : 0));
    {
        Dev d32, d16;
        if (d32.alloc(n * 4) != cudaSuccess || d16.alloc(n * 2) != cudaSuccess ||
            runOnDevice(s, d32.as<float>(), d16.as<unsigned short>()) != dh::ERR_SUCCESS ||
            cudaMemcpy(block, d32.p, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(b16, d16.p, n * 2, cudaMemcpyDeviceToHost) != cudaSuccess) {
            cudaGetLastError();
            free(block);
            return nullptr;
        }
    }
    // the resolved parameters, in the reference's order (digHolo.cpp:16074-16086)
    float* tX = prm;
    float* tY = tX + P;
    float* df = tY + P;
    float* rcx = df + P;
    float* rcy = rcx + P;
    float* rw = rcy + P;
    float* ra = rw + P;
    float* bw = ra + 2 * P;
    float* bcx = bw + P;
    float* bcy = bcx + P;
    float* bc = bcy + P;
    float* wl = bc + (size_t)s.frames * P * M * 2;
    for (int p = 0; p < P; p++) {
        tX[p] = s.tiltX[p];
        tY[p] = s.tiltY[p];
        df[p] = s.defocus[p];
        rcx[p] = s.refCx[p];
        rcy[p] = s.refCy[p];
        rw[p] = s.refWaist[p];
        ra[2 * p] = s.refAmp[p][0];
        ra[2 * p + 1] = s.refAmp[p][1];
        bw[p] = s.waist[p];
        bcx[p] = s.cx[p];
        bcy[p] = s.cy[p];
    }
    memcpy(bc, s.coefs.data(), s.coefs.size() * sizeof(float));
    memcpy(wl, s.wavelengths.data(), s.wavelengths.size() * sizeof(float));
    if (!*refTiltX) *refTiltX = tX;
    if (!*refTiltY) *refTiltY = tY;
    if (!*refDefocus) *refDefocus = df;
    if (!*refBeamCentreX) *refBeamCentreX = rcx;
    if (!*refBeamCentreY) *refBeamCentreY = rcy;
    if (!*refWaist) *refWaist = rw;
    if (!*refAmplitude) *refAmplitude = ra;
    if (!*beamWaist) *beamWaist = bw;
    if (!*beamCentreX) *beamCentreX = bcx;
    if (!*beamCentreY) *beamCentreY = bcy;
    if (!*beamCoefs) *beamCoefs = bc;
    if (!*wavelengths) *wavelengths = wl;
    *pixelBuffer16 = b16;
    if (fname) {
        FILE* f = fopen(fname, "wb");
        if (f) {
            fwrite(b16, sizeof(unsigned short), n, f);
            fclose(f);
        }
    }
    if (printToConsole) {
        printf("<FRAME SIMULATOR> %d frames %d x %d, %d polarisation(s), %d mode groups, %d levels, fill factor %d\n",
               s.frames, s.W, s.H, P, s.G, s.levels, s.fill);
        fflush(stdout);
    }
    return block;
}

// digHolo.h:2046
float* digHoloFrameSimulatorCreateSimple(int frameCount, int frameWidth, int frameHeight, float pixelSize, int polCount,
                                         float wavelength, int printToConsole) {
    if (frameWidth != QUANTA * (frameWidth / QUANTA) || frameHeight != QUANTA * (frameHeight / QUANTA)) return nullptr;
    if (frameCount < 1 || frameWidth < 1 || frameHeight < 1 || pixelSize <= 0 || polCount < 1 || wavelength <= 0)
        return nullptr;
    float *tX = nullptr, *tY = nullptr, *df = nullptr, *rw = nullptr, *rcx = nullptr, *rcy = nullptr, *ra = nullptr;
    float *bw = nullptr, *bc = nullptr, *bcx = nullptr, *bcy = nullptr;
    int G = 0, levels = 16384, L = 1;
    float* wl = &wavelength;
    unsigned short* b16 = nullptr;
    return digHoloFrameSimulatorCreate(frameCount, &frameWidth, &frameHeight, &pixelSize, &polCount, &tX, &tY, &df, &rw,
                                       &rcx, &rcy, &ra, &G, &bw, &bc, &bcx, &bcy, &levels, 1, &wl, &L, 0,
                                       printToConsole, &b16, nullptr);
}

// digHolo.h:2056
int digHoloFrameSimulatorDestroy(float* pixelBuffer) {
    if (!pixelBuffer) return dh::ERR_NULLPOINTER;
    free(pixelBuffer);
    return dh::ERR_SUCCESS;
}

// The simulator with its frames left in device memory (no host copy): the
// same parameters as digHoloFrameSimulatorCreate, given by value (null
// arrays take the same defaults); frames32 (device, frameCount x frameHeight
// x frameWidth float32, required: the intensities are formed there) and
// frames16 (device uint16, optional).  Frame sides must already be multiples
// of 16.  Returns a DIGHOLO_ERROR code.
int digHoloB200FrameSimulatorDevice(int frameCount, int frameWidth, int frameHeight, float pixelSize, int polCount,
                                    const float* refTiltX, const float* refTiltY, const float* refDefocus,
                                    const float* refWaist, const float* refBeamCentreX, const float* refBeamCentreY,
                                    int beamGroupCount, const float* beamWaist, const float* beamCoefs,
                                    const float* beamCentreX, const float* beamCentreY, int cameraPixelLevelCount,
                                    int fillFactorCorrection, const float* wavelengths, int wavelengthCount,
                                    float* frames32, unsigned short* frames16) {
    if (!frames32) return dh::ERR_NULLPOINTER;
    if (frameWidth % QUANTA || frameHeight % QUANTA) return dh::ERR_INVALIDDIMENSION;
    SimSpec s;
    int W = frameWidth, H = frameHeight, P = polCount, G = beamGroupCount, levels = cameraPixelLevelCount;
    int L = wavelengthCount;
    float ps = pixelSize;
    const int r = resolve(frameCount, W, H, ps, P, refTiltX, refTiltY, refDefocus, refWaist, refBeamCentreX,
                          refBeamCentreY, nullptr, G, beamWaist, beamCoefs, beamCentreX, beamCentreY, levels,
                          fillFactorCorrection, wavelengths, L, s);
    if (r != dh::ERR_SUCCESS) return r;
    return runOnDevice(s, frames32, frames16);
}

}  // extern "C"
