// Host runtime of digholo_b200: window geometry (float32 emulation of the
// reference), device buffer management, and the stage launches behind
// digHoloProcessBatch.
#include "dh_object.h"

#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cfloat>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

size_t dh_forward_smem_bytes(int logW, int logH, int colChunk);
cudaError_t dh_launch_forward(const DhFwdParams& p, cudaStream_t s);
cudaError_t dh_launch_forward_reg(const DhFwdParams& p, cudaStream_t s);
cudaError_t dh_launch_forward_tma(const DhFwdParams& p, cudaStream_t s);
cudaError_t dh_launch_forward_i8(const DhFwdParams& p, cudaStream_t s);
cudaError_t dh_launch_forward_i8_fused(const DhFwdParams& p, const DhInvParams& ip, cudaStream_t s);
cudaError_t dh_launch_fourier_full(const DhFourierParams& q, cudaStream_t s);
cudaError_t dh_launch_forward_plane(const DhFourierParams& q, cudaStream_t s);
size_t dh_field_band64_scratch_bytes(const DhInvParams& p, int overlapKind);
cudaError_t dh_launch_field_band64(const DhInvParams& p, int overlapKind, void* scratch, size_t scratchBytes,
                                   int* overlapUsed, cudaStream_t s);
int dh_forward_i8_npad(int w);
cudaError_t dh_launch_inverse_lo(const DhInvParams& p, cudaStream_t s);
cudaError_t dh_launch_field_full(const DhInvParams& p, int withOverlap, int* fused, cudaStream_t s);
cudaError_t dh_launch_overlap_f32(const DhInvParams& p, int nx, int ny, cudaStream_t s);
cudaError_t dh_launch_overlap_f32_chunked(const DhInvParams& p, int nx, int ny, cudaStream_t s);
size_t dh_field_big_scratch_bytes(const DhInvParams& p, int overlapKind);
cudaError_t dh_launch_field_big(const DhInvParams& p, int overlapKind, void* scratch, size_t scratchBytes,
                                int* overlapUsed, cudaStream_t s);
size_t dh_inverse_smem_bytes(const DhInvParams& p);
cudaError_t dh_launch_inverse(const DhInvParams& p, cudaStream_t s);
size_t dh_inverse_dft_smem_bytes(int w, int h, int G);
cudaError_t dh_launch_basis_transform(const float2* in, float2* out, const float2* T, int rows, int M, int din, int dout,
                                      cudaStream_t s);
cudaError_t dh_launch_inverse_dft(const DhInvParams& p, cudaStream_t s);
size_t dh_inverse_dft_global_bytes(const DhInvParams& p);
cudaError_t dh_launch_inverse_dft_global(const DhInvParams& p, void* scratch, size_t scratchBytes, cudaStream_t s);
cudaError_t dh_launch_basis(const DhBasisParams& p, cudaStream_t s);
cudaError_t dh_launch_untranspose_u16(const unsigned short* in, unsigned short* out, int Nx, int Ny, int frames,
                                      cudaStream_t s);
cudaError_t dh_launch_basis_jobs(const DhBasisParams* ps, int n, cudaStream_t s);
cudaError_t dh_launch_fields_to_c64(const short* R, const short* I, const float* stats, int statsStride,
                                    int polCount, int frameCount, int npix, float2* out, cudaStream_t s);
cudaError_t dh_launch_batchsum(const short* R, const short* I, const float* stats, int statsStride,
                               int polCount, int frameCount, int npix, float* out, cudaStream_t s);
cudaError_t dh_launch_average_windows(const float2* in, float2* out, int batch, int avg, int mode, int polCount,
                                      int n, const float2* cal, int calCount, cudaStream_t s);

namespace dh {

static const float PI_F = 3.14159265358979323846264338327950288f;   // digHolo.cpp:89
static const double PI_D = 3.14159265358979323846264338327950288;   // digHolo.cpp:3633
static const float UNIT_ANGLE = PI_F / 180.0f;                       // digHolo.h:192
static const int PIXEL_QUANTA = 16;                                  // digHolo.cpp:94

static std::atomic<unsigned long long> g_devBufGeneration{0};
unsigned long long devBufGeneration() { return g_devBufGeneration.load(std::memory_order_relaxed); }

cudaError_t DevBuf::ensure(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    if (n == 0) return cudaSuccess;
    g_devBufGeneration.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) { ptr = nullptr; bytes = 0; return e; }
    bytes = n;
    return cudaSuccess;
}
void DevBuf::release() {
    if (ptr) {
        g_devBufGeneration.fetch_add(1, std::memory_order_relaxed);
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
}
bool HostBuf::ensure(size_t n) {
    if (n <= bytes && ptr) return true;
    release();
    if (n == 0) return true;
    if (cudaMallocHost(&ptr, n) != cudaSuccess) { ptr = nullptr; bytes = 0; return false; }
    bytes = n;
    return true;
}
void HostBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

bool isPow2(int v) { return v > 0 && (v & (v - 1)) == 0; }
int ilog2(int v) { int l = 0; while ((1 << l) < v) l++; return l; }

// ------------------------------------------------------------------ geometry

static void axisShifted(int n, float step, std::vector<float>& a) {
    a.resize(n);
    for (int i = 0; i < n; i++) a[i] = step * (float)(i <= n / 2 ? i : i - n);
}
static void axisCentred(int n, float step, std::vector<float>& a) {
    a.resize(n);
    for (int i = 0; i < n; i++) a[i] = (float)(i - n / 2) * step;
}

// digHolo.cpp:7283-7378 and 7720-7733
void fftWindowGeometry(const Config& c, int P, Geometry& g) {
    const int fx = c.fftWindowSizeX > 0 ? c.fftWindowSizeX : c.frameWidth / P;
    const int fy = c.fftWindowSizeY > 0 ? c.fftWindowSizeY : c.frameHeight;
    int W = PIXEL_QUANTA * (fx / PIXEL_QUANTA);
    int H = PIXEL_QUANTA * (fy / PIXEL_QUANTA);
    W = std::max(W, 16);
    H = std::max(H, 16);
    W = std::min(W, c.frameWidth);
    H = std::min(H, c.frameHeight);
    const int block = 16;  // ALIGN / sizeof(float)
    for (int pol = 0; pol < P; pol++) {
        const float CX = (c.beamCentreX[pol] / c.pixelSize) + (float)(c.frameWidth / 2);
        const float CY = (c.beamCentreY[pol] / c.pixelSize) + (float)(c.frameHeight / 2);
        int cx = (int)std::round((CX - (float)(W / 2)) / (float)block) * block;
        int cy = (int)std::round(CY - (float)(H / 2));
        if (cx < 0) cx = 0;
        if (cy < 0) cy = 0;
        if (cx + W > c.frameWidth) cx = c.frameWidth - W;
        if (cy + H > c.frameHeight) cy = c.frameHeight - H;
        g.cx[pol] = cx;
        g.cy[pol] = cy;
    }
    g.W = W;
    g.H = H;
    const float period = (float)(2.0 * c.pixelSize);
    const float kfx = (float)(2 * (2.0 * PI_D / period) / W);
    const float kfy = (float)(2 * (2.0 * PI_D / period) / H);
    axisShifted(W, kfx, g.kx);
    axisShifted(H, kfy, g.ky);
    axisCentred(W, c.pixelSize, g.xFull);
    axisCentred(H, c.pixelSize, g.yFull);
}

// digHolo.cpp:7868-8048 (single wavelength) and 8183-8203
void ifftWindowGeometry(const Config& c, int P, Geometry& g) {
    // k0Max from the longest wavelength, k0Min from the shortest, as the
    // reference names them (digHolo.cpp:7913-7914)
    const float lamStart = c.lambdaRange[0] > 0 ? c.lambdaRange[0] : c.wavelengthCentre;
    const float lamStop = c.lambdaRange[1] > 0 ? c.lambdaRange[1] : c.wavelengthCentre;
    const float k0Max = 2 * PI_F / (fmaxf(lamStart, lamStop));
    const float k0Min = 2 * PI_F / (fminf(lamStart, lamStop));
    const float dkx = g.kx[1] - g.kx[0];
    const float dky = g.ky[1] - g.ky[0];
    const float r0 = c.apertureSize * UNIT_ANGLE;
    int woiCX[POLMAX], woiCY[POLMAX];
    int w = 0, h = 0;
    for (int pol = 0; pol < P; pol++) {
        const int src = c.polLockTilt ? 0 : pol;
        const float tx = c.zern[src][ZERN_TILTX] * UNIT_ANGLE;
        const float ty = c.zern[src][ZERN_TILTY] * UNIT_ANGLE;
        const float maxEX = (float)(((tx + r0) * k0Max) / dkx + g.W / 2.0);
        const float maxEY = (float)(((ty + r0) * k0Max) / dky + g.H / 2.0);
        const float minSX = (float)(((tx - r0) * k0Min) / dkx + g.W / 2.0);
        const float minSY = (float)(((ty - r0) * k0Min) / dky + g.H / 2.0);
        woiCX[pol] = (int)std::round((maxEX + minSX) / 4.0) * 2;
        woiCY[pol] = (int)std::round((maxEY + minSY) / 4.0) * 2;
        int wp = (int)(maxEX - minSX + 1);
        int hp = (int)(maxEY - minSY + 1);
        wp = (int)(16 * std::ceil((1.0f * wp) / 16));
        hp = (int)(16 * std::ceil((1.0f * hp) / 16));
        w = std::max(w, wp);
        h = std::max(h, hp);
    }
    if (h < 16) h = 16;
    if (w < 16) w = 16;
    for (int pol = 0; pol < P; pol++) {
        int sx = (int)(woiCX[pol] - w / 2.0);
        if (sx < g.W / 2) sx = g.W / 2;
        if (sx < 0) sx = 0;
        if (sx + w > g.W) sx = g.W - w;
        g.SX[pol] = sx;
        g.SY[pol] = (int)(woiCY[pol] - h / 2.0);
    }
    g.w = w;
    g.h = h;
    const int nx = c.resolutionIdx ? w : g.W;
    const int ny = c.resolutionIdx ? h : g.H;
    g.nx = nx;
    g.ny = ny;
    const float psx = ((c.pixelSize) * g.W) / nx;
    const float psy = ((c.pixelSize) * g.H) / ny;
    axisCentred(nx, psx, g.x);
    axisCentred(ny, psy, g.y);
}

// Separable 14-bit reference wave per polarisation (digHolo.cpp:10201-10504):
// out[pol][0..nx) Xr, [nx..2nx) Xi, [2nx..2nx+ny) Yr, [2nx+ny..) Yi.
void referenceWave(const Config& c, int P, const Geometry& g, std::vector<short>& out, std::vector<float>* outF) {
    const int nx = g.nx, ny = g.ny;
    if (outF) outF->assign((size_t)P * 2 * (nx + ny), 0.f);
    const std::vector<float>& xa = c.resolutionIdx ? g.x : g.xFull;
    const std::vector<float>& ya = c.resolutionIdx ? g.y : g.yFull;
    out.assign((size_t)P * 2 * (nx + ny), 0);
    const float dkx = g.kx[1] - g.kx[0];
    const float dky = g.ky[1] - g.ky[0];
    for (int pol = 0; pol < P; pol++) {
        const int st = c.polLockTilt ? 0 : pol;
        const int sd = c.polLockDefocus ? 0 : pol;
        const float tx = c.zern[st][ZERN_TILTX] * UNIT_ANGLE;
        const float ty = c.zern[st][ZERN_TILTY] * UNIT_ANGLE;
        float offx = 0.f, offy = 0.f;
        if (c.resolutionIdx == 1) {
            offx = (float)((g.SX[st] - g.W / 2.0 - 0) * dkx);
            offy = (float)((g.SY[st] - g.H / 2.0) * dky);
        }
        const float dioptre = c.zern[sd][ZERN_DEFOCUS];
        const float lam = c.wavelengthCentre;
        const float k0 = (float)(2.0 * PI_F / lam);
        const float kx = -k0 * tx + offx;
        const float ky = -k0 * ty + offy;
        const float kx0 = offx == 0 ? kx : k0 * (-tx);
        const float ky0 = offy == 0 ? ky : k0 * (-ty);
        const float focal = (float)(-PI_F * dioptre / lam);
        const float pistX = c.beamCentreX[pol] * kx0;
        const float pistY = c.beamCentreY[pol] * ky0;
        short* o = &out[(size_t)pol * 2 * (nx + ny)];
        for (int axis = 0; axis < 2; axis++) {
            const std::vector<float>& a = axis == 0 ? xa : ya;
            const int n = axis == 0 ? nx : ny;
            const float k = axis == 0 ? kx : ky;
            const float piston = axis == 0 ? pistX : pistY;
            short* re = axis == 0 ? o : o + 2 * nx;
            short* im = axis == 0 ? o + nx : o + 2 * nx + ny;
            for (int i = 0; i < n; i++) {
                const float r = a[i];
                const float kr = std::fma(k, r, piston);
                const float arg = kr + focal * (r * r);
                const float cs = (float)std::cos((double)arg);
                const float sn = (float)std::sin((double)arg);
                const float vr = std::nearbyint(16383.0f * cs);
                const float vi = std::nearbyint(16383.0f * sn);
                re[i] = (short)std::max(-32768.f, std::min(32767.f, vr));
                im[i] = (short)std::max(-32768.f, std::min(32767.f, vi));
                if (outF) {
                    float* f = outF->data() + (size_t)pol * 2 * (nx + ny) + (re - o);
                    f[i] = cs;
                    f[i + (im - re)] = sn;
                }
            }
        }
    }
}

// ------------------------------------------------------------------ device

int objInitDevice(Object& o) {
    if (o.device >= 0) {
        cudaSetDevice(o.device);
        return ERR_SUCCESS;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(o, ERR_ERROR, "no CUDA device available: digholo_b200 runs on the GPU only");
    int dev = 0;
    DH_CUDA(o, cudaGetDevice(&dev));
    o.device = dev;
    if (!o.stream) DH_CUDA(o, cudaStreamCreateWithFlags(&o.stream, cudaStreamNonBlocking));
    DH_CUDA(o, cudaStreamCreateWithFlags(&o.copyStream, cudaStreamNonBlocking));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evCopy[0], cudaEventDisableTiming));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evCopy[1], cudaEventDisableTiming));
    DH_CUDA(o, cudaStreamCreateWithFlags(&o.copyStream2, cudaStreamNonBlocking));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evCopy2[0], cudaEventDisableTiming));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evCopy2[1], cudaEventDisableTiming));
    DH_CUDA(o, cudaStreamCreateWithFlags(&o.d2hStream, cudaStreamNonBlocking));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evChunk[0], cudaEventDisableTiming));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evChunk[1], cudaEventDisableTiming));
    DH_CUDA(o, cudaEventCreateWithFlags(&o.evD2H, cudaEventDisableTiming));
    DH_CUDA(o, cudaEventCreate(&o.evStart));
    DH_CUDA(o, cudaEventCreate(&o.evStop));
    // twiddle(k) = exp(-2 pi i k / 4096), double precision rounded to float
    std::vector<float> tw(2 * 4096);
    for (int k = 0; k < 4096; k++) {
        const double a = -2.0 * PI_D * (double)k / 4096.0;
        tw[2 * k] = (float)std::cos(a);
        tw[2 * k + 1] = (float)std::sin(a);
    }
    DH_CUDA(o, o.dTwiddle.ensure(tw.size() * sizeof(float)));
    DH_CUDA(o, cudaMemcpy(o.dTwiddle.ptr, tw.data(), tw.size() * sizeof(float), cudaMemcpyHostToDevice));
    DH_CUDA(o, cudaHostAlloc(reinterpret_cast<void**>(&o.hStatus), sizeof(int), cudaHostAllocMapped));
    *o.hStatus = 0;
    DH_CUDA(o, cudaHostGetDevicePointer(reinterpret_cast<void**>(&o.dStatus), o.hStatus, 0));
    return ERR_SUCCESS;
}

static int isDevicePointer(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Checks the configuration against what the fused kernels support.
static int checkSupported(Object& o) {
    const Geometry& g = o.geo;
    if (!isPow2(g.W) || !isPow2(g.H) || g.W > 2048 || g.H > 2048)
        return fail(o, ERR_INVALIDDIMENSION, "FFT window sides must be powers of two up to 2048 on this build");
    // IFFT windows whose sides are multiples of 16 but not powers of two:
    // the full-plane forward, then at full resolution the band kernels (FFT
    // windows of at least 64 x 64), in low-resolution mode the DFT kernel
    // (its planes in shared memory up to about 112 x 112 with 15 mode
    // groups, in global scratch beyond)
    if (!isPow2(g.w) || !isPow2(g.h)) {
        const bool m16 = g.w % 16 == 0 && g.h % 16 == 0;
        const bool bands = o.cfg.resolutionIdx == 0 && g.W >= 64 && g.H >= 64 && m16;
        const bool dft = o.cfg.resolutionIdx != 0 && m16;
        if (!bands && !dft)
            return fail(o, ERR_INVALIDDIMENSION,
                        "IFFT window sides that are not powers of two need an FFT window of at least 64 x 64 at full "
                        "resolution on this build");
    }
    if (o.avgCount < 1 || o.cfg.avgMode < 0 || o.cfg.avgMode > 2)
        return fail(o, ERR_INVALIDARGUMENT, "frame averaging: avgCount must be at least 1 and avgMode 0, 1 or 2");
    return ERR_SUCCESS;
}

static int colChunkFor(const Geometry& g) {
    // Keep the column buffer of the forward kernel within 128 KB.
    int wc = g.w;
    while ((size_t)g.H * wc * sizeof(float2) > 128 * 1024 && wc > 1) wc >>= 1;
    return wc;
}

// Resolve the frame source for frames [f0, f1): device pointer in place, or
// a strided copy of the FFT windows from host memory into the staging buffer.
static int stageFrames(Object& o, int f0, int f1, DhFwdParams& fp, int async) {
    const Geometry& g = o.geo;
    const int P = o.polCount;
    const size_t es = o.framesU16 ? 2 : 4;
    if (o.framesOnDevice) {
        fp.frames = o.frames;
        fp.frameWidth = o.cfg.frameWidth;
        fp.frameStride = (long long)o.cfg.frameWidth * o.cfg.frameHeight;
        for (int p = 0; p < P; p++) { fp.cx[p] = g.cx[p]; fp.cy[p] = g.cy[p]; }
        return ERR_SUCCESS;
    }
    const size_t frameBytes = (size_t)P * g.H * g.W * es;
    DH_CUDA(o, o.dFrames.ensure(frameBytes * (size_t)o.batchCount * std::max(1, o.avgCount)));
    for (int p = 0; p < P; p++) {
        cudaMemcpy3DParms m;
        memset(&m, 0, sizeof(m));
        m.srcPtr = make_cudaPitchedPtr(const_cast<void*>(o.frames), (size_t)o.cfg.frameWidth * es,
                                       (size_t)o.cfg.frameWidth * es, (size_t)o.cfg.frameHeight);
        m.srcPos = make_cudaPos((size_t)g.cx[p] * es, (size_t)g.cy[p], (size_t)f0);
        m.dstPtr = make_cudaPitchedPtr(o.dFrames.ptr, (size_t)g.W * es, (size_t)g.W * es, (size_t)P * g.H);
        m.dstPos = make_cudaPos(0, (size_t)p * g.H, (size_t)f0);
        m.extent = make_cudaExtent((size_t)g.W * es, (size_t)g.H, (size_t)(f1 - f0));
        m.kind = cudaMemcpyHostToDevice;
        DH_CUDA(o, cudaMemcpy3DAsync(&m, async ? ((p & 1) ? o.copyStream2 : o.copyStream) : o.stream));
    }
    fp.frames = o.dFrames.ptr;
    fp.frameWidth = g.W;
    fp.frameStride = (long long)P * g.H * g.W;
    for (int p = 0; p < P; p++) { fp.cx[p] = 0; fp.cy[p] = p * g.H; }
    return ERR_SUCCESS;
}

// Window factors of digHoloCopyWindow (digHolo.cpp:1955-2035) per
// polarisation, [pol][h][w] complex: the hard mask dr^2 <= kr^2 around the
// tilt, the inverse pixel sinc, the normalisation 1/sqrt(W H . ifft length)
// and the beam-centre phase exp(i (kx bcx + ky bcy)), in the reference's
// float32 arithmetic.  `c` places the window and the mask, `live` gives the
// beam centre (the two differ while AutoAlign replays stage snapshots).
void windowFactors(const Config& c, const Config& live, const Geometry& g, int P, std::vector<float>& adj) {
    const int w = g.w, h = g.h, W = g.W, H = g.H;
    adj.assign((size_t)P * h * w * 2, 0.f);
    const float lam = c.wavelengthCentre;
    const float k0 = 2 * PI_F / lam;
    const float kr = k0 * sinf(c.apertureSize * UNIT_ANGLE);
    const float r02 = kr * kr;
    const double fftLength = 1.0 * W * H;
    const double ifftLength = c.resolutionIdx ? 1.0 * w * h : fftLength;
    const float norm = (float)(1.0 / sqrt(fftLength * ifftLength));
    const float halfPixel = 0.5f * c.pixelSize;
    const float kyShift = fabsf((g.ky[1] - g.ky[0]) * H);
    auto xcscD = [](float x) { return x == 0.f ? 1.0f : (float)((double)x / sin((double)x)); };
    for (int p = 0; p < P; p++) {
        const int sx0 = g.SX[p] - W / 2;
        const int cx0 = (g.cx[p] + W / 2) - c.frameWidth / 2;
        const int cy0 = (g.cy[p] + H / 2) - c.frameHeight / 2;
        const float bcx = live.beamCentreX[p] - (cx0) * c.pixelSize;
        const float bcy = live.beamCentreY[p] - (cy0) * c.pixelSize;
        const float kx0 = k0 * sinf(c.zern[p][ZERN_TILTX] * UNIT_ANGLE);
        const float ky0 = k0 * sinf(c.zern[p][ZERN_TILTY] * UNIT_ANGLE);
        for (int j = 0; j < h; j++) {
            const int jSY = j + g.SY[p];
            int row = (jSY + H / 2) % H;
            if (row < 0) row += H;
            const float ky = g.ky[row];
            const float shift = jSY < 0 ? kyShift : (jSY > H ? -kyShift : 0.0f);
            for (int cc = 0; cc < w; cc++) {
                const float kx = g.kx[sx0 + cc];
                volatile float dky = ky - (ky0 + shift);
                volatile float dkx = kx - kx0;
                volatile float dkx2 = dkx * dkx;
                volatile float dky2 = dky * dky;
                const float dr2 = dkx2 + dky2;
                const float env = c.fillFactorCorrection ? xcscD(kx * halfPixel) * xcscD(ky * halfPixel) : 1.0f;
                const float normF = (dr2 <= r02) ? env * norm : 0.0f;
                volatile float ax = bcx * kx;
                volatile float ay = ky * bcy;
                const float arg = ax + ay;
                const size_t o2 = (((size_t)p * h + j) * w + cc) * 2;
                adj[o2] = (float)cos((double)arg) * normF;
                adj[o2 + 1] = (float)sin((double)arg) * normF;
            }
        }
    }
}

// Frame-independent factors of the forward stage for the register kernel,
// evaluated with the float32 arithmetic of digHoloCopyWindow
// (digHolo.cpp:1955-2035): per polarisation, the R2C split twiddles
// [w], the column-sum twiddles [h][H/h] and the window factors [h][w].
static void forwardTables(const Object& o, std::vector<float>& split, std::vector<float>& col,
                          std::vector<float>& adj) {
    const Config& c = o.useSnaps ? o.ifftSnap : o.cfg;
    const Geometry& g = o.geo;
    const int P = o.polCount, w = g.w, h = g.h, W = g.W, H = g.H;
    const int Q = H / h;
    split.assign((size_t)P * w * 2, 0.f);
    col.assign((size_t)P * h * Q * 2, 0.f);
    for (int p = 0; p < P; p++) {
        const int sx0 = g.SX[p] - W / 2;
        for (int cc = 0; cc < w; cc++) {
            const double a = -2.0 * PI_D * (double)(sx0 + cc) / (double)W;
            split[((size_t)p * w + cc) * 2] = (float)cos(a);
            split[((size_t)p * w + cc) * 2 + 1] = (float)sin(a);
        }
        for (int j = 0; j < h; j++) {
            const int jSY = j + g.SY[p];
            int row = (jSY + H / 2) % H;
            if (row < 0) row += H;
            for (int b = 0; b < Q; b++) {
                const double a = -2.0 * PI_D * (double)((row * b) % H) / (double)H;
                col[(((size_t)p * h + j) * Q + b) * 2] = (float)cos(a);
                col[(((size_t)p * h + j) * Q + b) * 2 + 1] = (float)sin(a);
            }
        }
    }
    // the beam-centre phase follows the live configuration; the window
    // selection and the mask may come from a snapshot
    windowFactors(c, o.cfg, g, P, adj);
}

// Byte digits of the tensor-core row DFT (k_forward_i8): for every kept kx
// column k = sx0 + c the 22-bit fixed-point values v = round((cos(2 pi k x / W)
// + 1) 2^22) and round((1 - sin(2 pi k x / W)) 2^22), v = d0 2^16 + d1 2^8 +
// d2, and a ones column (v = 1).  Accumulator q pairs the low byte of pixel x
// with digit q - 1 and the high byte with digit q (digits -1 and 3 are zero).
// Layout [pol][atom][4 npad][128 B] (row q npad + n: the four accumulators'
// operands stacked along N), 16-byte chunk c of row n at c ^ (n & 7) (the
// K-major 128-byte-swizzled operand; npad is a multiple of 8).  Empty when the kernel does not
// apply to the geometry.
static void dftDigits(const Object& o, std::vector<unsigned char>& out) {
    out.clear();
    const Geometry& g = o.geo;
    const int W = g.W, w = g.w, P = o.polCount;
    if (!o.framesU16 || g.H != 128 || (W != 64 && W != 128) || g.h != w || (w != 16 && w != 32)) return;
    const int npad = dh_forward_i8_npad(w), natom = 2 * W / 128;
    out.assign((size_t)P * 4 * natom * npad * 128, 0);
    for (int p = 0; p < P; p++) {
        const int sx0 = g.SX[p] - W / 2;
        for (int n = 0; n < npad; n++) {
            for (int x = 0; x < W; x++) {
                long long v = 0;
                if (n < 2 * w) {
                    const int k = sx0 + (n < w ? n : n - w);
                    const int m = (int)((((long long)k * x) % W + W) % W);
                    const double ang = 2.0 * PI_D * (double)m / (double)W;
                    const double val = n < w ? cos(ang) + 1.0 : 1.0 - sin(ang);
                    v = llround(val * 4194304.0);
                } else if (n == 2 * w) {
                    v = 1;
                }
                const unsigned char d[3] = {(unsigned char)(v >> 16), (unsigned char)((v >> 8) & 255),
                                            (unsigned char)(v & 255)};
                for (int q = 0; q < 4; q++) {
                    for (int hi = 0; hi < 2; hi++) {
                        const int di = q - 1 + hi;
                        const unsigned char byte = (di >= 0 && di <= 2) ? d[di] : 0;
                        const int b = 2 * x + hi, a = b >> 7, bb = b & 127, ch = bb >> 4;
                        const size_t off = (((size_t)p * natom + a) * 4 * npad + (size_t)q * npad + n) * 128 +
                                           (size_t)((ch ^ (n & 7)) << 4) + (bb & 15);
                        out[off] = byte;
                    }
                }
            }
        }
    }
}

static void forwardParams(Object& o, DhFwdParams& fp) {
    const Config& c = o.useSnaps ? o.ifftSnap : o.cfg;
    const Geometry& g = o.geo;
    memset(&fp, 0, sizeof(fp));
    fp.inputU16 = o.framesU16;
    fp.polCount = o.polCount;
    fp.logW = ilog2(g.W);
    fp.logH = ilog2(g.H);
    fp.w = g.w;
    fp.h = g.h;
    fp.colChunk = colChunkFor(g);
    const float lam = c.wavelengthCentre;
    const float k0 = 2 * PI_F / lam;                       // digHolo.cpp:8626
    const float ap = c.apertureSize * UNIT_ANGLE;
    const float kr = k0 * sinf(ap);
    for (int p = 0; p < o.polCount; p++) {
        fp.sx0[p] = g.SX[p] - g.W / 2;
        fp.sy[p] = g.SY[p];
        const int cx0 = (g.cx[p] + g.W / 2) - c.frameWidth / 2;   // digHolo.cpp:8580-8584
        const int cy0 = (g.cy[p] + g.H / 2) - c.frameHeight / 2;
        fp.bcx[p] = o.cfg.beamCentreX[p] - (cx0) * c.pixelSize;
        fp.bcy[p] = o.cfg.beamCentreY[p] - (cy0) * c.pixelSize;
        const float tx = c.zern[p][ZERN_TILTX] * UNIT_ANGLE;       // digHolo.cpp:8588-8589
        const float ty = c.zern[p][ZERN_TILTY] * UNIT_ANGLE;
        fp.kx0[p] = k0 * sinf(tx);
        fp.ky0[p] = k0 * sinf(ty);
        fp.r02[p] = kr * kr;
    }
    fp.kyShift = fabsf((g.ky[1] - g.ky[0]) * g.H);
    const double fftLength = 1.0 * g.W * g.H;
    const double ifftLength = c.resolutionIdx ? 1.0 * g.w * g.h : fftLength;
    fp.norm = (float)(1.0 / sqrt(fftLength * ifftLength));
    fp.halfPixel = 0.5f * c.pixelSize;
    fp.fillFactor = c.fillFactorCorrection;
    fp.kxAxis = o.dKx.as<float>();
    fp.kyAxis = o.dKy.as<float>();
    if (o.batchCalEnabled && o.batchCalCount > 0 && o.dBatchCal.ptr) {
        fp.batchCal = o.dBatchCal.as<float2>();
        fp.batchCalCount = o.batchCalCount;
    }
    fp.window = o.dWindow.as<float2>();
    fp.twiddle = o.dTwiddle.as<float2>();
    fp.status = o.dStatus;
    if (o.dTables.ptr) {
        const Geometry& gg = o.geo;
        const size_t P = o.polCount;
        float2* t = o.dTables.as<float2>();
        fp.tabSplit = t;
        fp.tabCol = t + P * gg.w;
        fp.tabAdj = t + P * gg.w + P * gg.h * (gg.H / gg.h);
    }
    if (o.digitsValid && o.dDigits.ptr) {
        fp.dftDigits = o.dDigits.as<unsigned char>();
        fp.dftNpad = o.digitsValid;
    }
}

// digHoloFFT_SetWindow + digHoloIFFT_SetWindow: geometry, axes, buffers.
static int prepare(Object& o) {
    int r = objInitDevice(o);
    if (r) return r;
    Config& c = o.cfg;
    if (!o.frames) return fail(o, ERR_NULLPOINTER, "frame buffer not set");
    if (c.batchCount <= 0) c.batchCount = 1;
    o.batchCount = c.batchCount;
    o.avgCount = c.avgCount;
    o.polCount = c.polCount;
    // the reference stores the default window size back into the config (digHolo.cpp:7283-7290)
    if (c.fftWindowSizeX <= 0) c.fftWindowSizeX = c.frameWidth / c.polCount;
    if (c.fftWindowSizeY <= 0) c.fftWindowSizeY = c.frameHeight;
    // an unchanged configuration keeps its geometry, tables and buffers
    const bool unchanged = !o.useSnaps && o.preparedValid && memcmp(&o.preparedCfg, &c, sizeof(Config)) == 0 &&
                           o.preparedKeep32 == o.keepField32 && o.preparedU16 == o.framesU16 &&
                           o.preparedBatchCal == o.batchCalVersion;
    if (!unchanged) {
        // AutoAlign evaluations place the FFT and IFFT windows with the settings of
        // the last evaluation that reran those stages (stage snapshots)
        fftWindowGeometry(o.useSnaps ? o.fftSnap : c, o.polCount, o.geo);
        ifftWindowGeometry(o.useSnaps ? o.ifftSnap : c, o.polCount, o.geo);
        r = checkSupported(o);
        if (r) return r;
    }
    const Geometry& g = o.geo;
    if (!o.framesOnDevice) {
        o.framesOnDevice = isDevicePointer(o.frames);
    }
    if (o.framesOnDevice) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(o.frames);
        if (a % 16) return fail(o, ERR_INVALIDARGUMENT, "device frame buffer must be 16-byte aligned");
    }
    if (unchanged) return ERR_SUCCESS;
    o.preparedValid = 0;
    // Uploads go through one pinned staging buffer; its previous contents
    // must have left before it is rewritten (no stream-wide synchronisation).
    if (o.evUpload) DH_CUDA(o, cudaEventSynchronize(o.evUpload));
    std::vector<float> split, col, adj;
    forwardTables(o, split, col, adj);
    std::vector<unsigned char> digits;
    dftDigits(o, digits);
    std::vector<short> ref;
    std::vector<float> refF;
    referenceWave(c, o.polCount, g, ref, &refF);
    const size_t nUp = (size_t)g.W + g.H + g.nx + g.ny + 2 * (split.size() + col.size() + adj.size()) + refF.size() +
                       (ref.size() + 1) / 2 + (o.batchCalEnabled ? o.batchCal.size() : 0) + digits.size() / 4 + 64;
    if (!o.hUpload.ensure(nUp * sizeof(float))) return fail(o, ERR_MEMORYALLOCATION, "pinned upload buffer");
    float* up = o.hUpload.as<float>();
    size_t upOff = 0;
    auto stage = [&](DevBuf& dst, const void* src, size_t bytes) -> int {
        DH_CUDA(o, dst.ensure(bytes));
        memcpy(up + upOff, src, bytes);
        DH_CUDA(o, cudaMemcpyAsync(dst.ptr, up + upOff, bytes, cudaMemcpyHostToDevice, o.stream));
        upOff += (bytes + sizeof(float) - 1) / sizeof(float);
        return ERR_SUCCESS;
    };
    if ((r = stage(o.dKx, g.kx.data(), g.W * sizeof(float)))) return r;
    if ((r = stage(o.dKy, g.ky.data(), g.H * sizeof(float)))) return r;
    if ((r = stage(o.dX, g.x.data(), g.nx * sizeof(float)))) return r;
    if ((r = stage(o.dY, g.y.data(), g.ny * sizeof(float)))) return r;
    const size_t B = (size_t)o.batchCount, P = (size_t)o.polCount;
    DH_CUDA(o, o.dWindow.ensure(B * P * g.w * g.h * sizeof(float2)));
    const size_t npix = (size_t)g.nx * g.ny;
    DH_CUDA(o, o.dFieldR.ensure(B * P * npix * sizeof(short)));
    DH_CUDA(o, o.dFieldI.ensure(B * P * npix * sizeof(short)));
    if (o.keepField32) DH_CUDA(o, o.dField32.ensure(B * P * npix * sizeof(float2)));
    DH_CUDA(o, o.dStats.ensure((size_t)ANALYSIS_COUNT * P * (B + 1) * sizeof(float)));
    if (o.batchCalEnabled && o.batchCalCount > 0) {
        if ((r = stage(o.dBatchCal, o.batchCal.data(), o.batchCal.size() * sizeof(float)))) return r;
    }
    {
        // tables: split, column-sum and window factors, contiguous on the device
        std::vector<float> tabs;
        tabs.reserve(split.size() + col.size() + adj.size());
        tabs.insert(tabs.end(), split.begin(), split.end());
        tabs.insert(tabs.end(), col.begin(), col.end());
        tabs.insert(tabs.end(), adj.begin(), adj.end());
        if ((r = stage(o.dTables, tabs.data(), tabs.size() * sizeof(float)))) return r;
    }
    o.digitsValid = 0;
    if (!digits.empty()) {
        if ((r = stage(o.dDigits, digits.data(), digits.size()))) return r;
        o.digitsValid = dh_forward_i8_npad(g.w);
    }
    // reference wave (cheap to recompute on the host)
    if ((r = stage(o.dRef, ref.data(), ref.size() * sizeof(short)))) return r;
    if ((r = stage(o.dRefF, refF.data(), refF.size() * sizeof(float)))) return r;
    if (!o.evUpload) DH_CUDA(o, cudaEventCreateWithFlags(&o.evUpload, cudaEventDisableTiming));
    DH_CUDA(o, cudaEventRecord(o.evUpload, o.stream));
    o.preparedCfg = c;
    o.preparedKeep32 = o.keepField32;
    o.preparedU16 = o.framesU16;
    o.preparedBatchCal = o.batchCalVersion;
    o.preparedValid = o.useSnaps ? 0 : 1;
    return ERR_SUCCESS;
}

// HG basis on the reconstructed-plane axes (digHolo.cpp:10506-10645).
static int updateBasis(Object& o) {
    Config& c = o.cfg;
    const Geometry& g = o.geo;
    const int G = c.maxMG;
    const int P = o.polCount;
    if (G <= 0) { o.modeCount = 0; return ERR_SUCCESS; }
    float waist[POLMAX] = {c.waist[0], c.waist[1]};
    for (int p = 0; p < P; p++) if (waist[p] == 0) waist[p] = 400e-6f;
    if (c.polLockBasisWaist) { waist[1] = waist[0]; c.waist[1] = c.waist[0]; }
    const std::vector<float>& xa = c.resolutionIdx ? g.x : g.xFull;
    const std::vector<float>& ya = c.resolutionIdx ? g.y : g.yFull;
    const float psx = xa[1] - xa[0];
    const float psy = ya[1] - ya[0];
    o.modeCount = G * (G + 1) / 2;
    if (o.basisNx == g.nx && o.basisNy == g.ny && o.basisMG == G && o.basisPolCount == P &&
        o.basisWaist[0] == waist[0] && o.basisWaist[1] == waist[1] && o.basisPsx == psx && o.basisPsy == psy)
        return ERR_SUCCESS;
    const int nx = g.nx, ny = g.ny;
    DH_CUDA(o, o.dHgX.ensure((size_t)P * G * nx * sizeof(short)));
    DH_CUDA(o, o.dHgY.ensure((size_t)P * G * ny * sizeof(short)));
    DH_CUDA(o, o.dHgScaleX.ensure((size_t)P * G * sizeof(float)));
    DH_CUDA(o, o.dHgScaleY.ensure((size_t)P * G * sizeof(float)));
    const bool square = (psx == psy);
    const int L = std::max(nx, ny);
    DH_CUDA(o, o.dBasisAxis.ensure((size_t)(nx + ny + L) * sizeof(float) + (size_t)G * L * sizeof(short)));
    float* dAxis = o.dBasisAxis.as<float>();
    short* dLong = reinterpret_cast<short*>(dAxis + nx + ny + L);
    for (int p = 0; p < P; p++) {
        const int src = (P > 1 && waist[1] == waist[0]) ? 0 : p;
        short* hx = o.dHgX.as<short>() + (size_t)p * G * nx;
        short* hy = o.dHgY.as<short>() + (size_t)p * G * ny;
        float* sx = o.dHgScaleX.as<float>() + (size_t)p * G;
        float* sy = o.dHgScaleY.as<float>() + (size_t)p * G;
        if (src != p) {
            DH_CUDA(o, cudaMemcpyAsync(hx, o.dHgX.as<short>(), (size_t)G * nx * sizeof(short), cudaMemcpyDeviceToDevice, o.stream));
            DH_CUDA(o, cudaMemcpyAsync(hy, o.dHgY.as<short>(), (size_t)G * ny * sizeof(short), cudaMemcpyDeviceToDevice, o.stream));
            DH_CUDA(o, cudaMemcpyAsync(sx, o.dHgScaleX.as<float>(), (size_t)G * sizeof(float), cudaMemcpyDeviceToDevice, o.stream));
            DH_CUDA(o, cudaMemcpyAsync(sy, o.dHgScaleY.as<float>(), (size_t)G * sizeof(float), cudaMemcpyDeviceToDevice, o.stream));
            continue;
        }
        if (square) {
            // one set of modes on the longer axis; the shorter axis reads its centred sub-range
            const std::vector<float>& la = nx >= ny ? xa : ya;
            DH_CUDA(o, cudaMemcpyAsync(dAxis, la.data(), L * sizeof(float), cudaMemcpyHostToDevice, o.stream));
            DhBasisParams bp{dAxis, L, G, (double)waist[p], dLong, sx, nullptr, G};
            DH_CUDA(o, dh_launch_basis(bp, o.stream));
            DH_CUDA(o, cudaMemcpyAsync(sy, sx, (size_t)G * sizeof(float), cudaMemcpyDeviceToDevice, o.stream));
            const int off = (L - std::min(nx, ny)) / 2;
            const int offX = nx >= ny ? 0 : off;
            const int offY = nx >= ny ? off : 0;
            DH_CUDA(o, cudaMemcpy2DAsync(hx, nx * sizeof(short), dLong + offX, L * sizeof(short), nx * sizeof(short), G,
                                         cudaMemcpyDeviceToDevice, o.stream));
            DH_CUDA(o, cudaMemcpy2DAsync(hy, ny * sizeof(short), dLong + offY, L * sizeof(short), ny * sizeof(short), G,
                                         cudaMemcpyDeviceToDevice, o.stream));
        } else {
            DH_CUDA(o, cudaMemcpyAsync(dAxis, xa.data(), nx * sizeof(float), cudaMemcpyHostToDevice, o.stream));
            DH_CUDA(o, cudaMemcpyAsync(dAxis + nx, ya.data(), ny * sizeof(float), cudaMemcpyHostToDevice, o.stream));
            DhBasisParams bx{dAxis, nx, G, (double)waist[p], hx, sx, nullptr, G};
            DH_CUDA(o, dh_launch_basis(bx, o.stream));
            DhBasisParams by{dAxis + nx, ny, G, (double)waist[p], hy, sy, nullptr, G};
            DH_CUDA(o, dh_launch_basis(by, o.stream));
        }
        DH_CUDA(o, cudaStreamSynchronize(o.stream));
    }
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    o.basisNx = nx; o.basisNy = ny; o.basisMG = G; o.basisPolCount = P;
    o.basisWaist[0] = waist[0]; o.basisWaist[1] = waist[1];
    o.basisPsx = psx; o.basisPsy = psy;
    return ERR_SUCCESS;
}

// HG basis for the current configuration (recomputed when the waist, axes or
// group count changed); the benchmark forces one recomputation.
int objUpdateBasis(Object& o) {
    std::lock_guard<std::mutex> guard(o.lock);
    return updateBasis(o);
}

static void inverseParams(Object& o, DhInvParams& ip, int withOverlap) {
    const Geometry& g = o.geo;
    memset(&ip, 0, sizeof(ip));
    ip.window = o.dWindow.as<float2>();
    ip.frameCount = o.batchCount;
    ip.polCount = o.polCount;
    ip.lowres = o.cfg.resolutionIdx;
    ip.logW = ilog2(g.W); ip.logH = ilog2(g.H);
    ip.logw = ilog2(g.w); ip.logh = ilog2(g.h);
    ip.w = g.w; ip.h = g.h;
    for (int p = 0; p < o.polCount; p++) { ip.sx0[p] = g.SX[p] - g.W / 2; ip.sy[p] = g.SY[p]; }
    ip.refWave = o.dRef.as<short>();
    ip.refWaveF = o.dRefF.as<float>();
    ip.status = o.dStatus;
    ip.xAxis = o.dX.as<float>();
    ip.yAxis = o.dY.as<float>();
    ip.dA = fabsf(g.x[2] - g.x[1]) * fabsf(g.y[2] - g.y[1]);
    ip.fieldR = o.dFieldR.as<short>();
    ip.fieldI = o.dFieldI.as<short>();
    ip.field32 = o.keepField32 ? o.dField32.as<float2>() : nullptr;
    ip.stats = o.dStats.as<float>();
    ip.statsStride = o.batchCount + 1;
    if (withOverlap && o.modeCount > 0) {
        ip.maxMG = o.cfg.maxMG;
        ip.modeCount = o.modeCount;
        ip.hgX = o.dHgX.as<short>();
        ip.hgY = o.dHgY.as<short>();
        ip.hgScaleX = o.dHgScaleX.as<float>();
        ip.hgScaleY = o.dHgScaleY.as<float>();
        ip.coefs = o.dCoefs.as<float2>();
    }
    ip.twiddle = o.dTwiddle.as<float2>();
}

// The reference-wave calibration planes of this batch, where a calibration
// applies (digHolo.cpp:8242-8246); lookupOnly: planes computed by an earlier
// batch only (nothing is allocated).
static int calParams(Object& o, DhInvParams& ip, bool lookupOnly = false) {
    if (!objRefCalApplies(o)) return ERR_SUCCESS;
    int r = objRefCalCheckShape(o, ip);
    if (r) return r;
    const float2* planes = nullptr;
    r = objRefCalPlanes(o, o.sweepLambda >= 0 ? o.sweepLambda : 0, &planes, lookupOnly);
    if (r) return r;
    ip.refCal = planes;
    return ERR_SUCCESS;
}

// Forward stage: the TMA-fed persistent kernel where the shape and the
// alignment allow it, else the register kernel, else the generic one.
static cudaError_t launchForward(Object& o, const DhFwdParams& fp, bool mayAlloc = true) {
    const int mode = o.forwardKernel;
    cudaError_t fe = cudaErrorNotSupported;
    if (mode == 0 || mode == 4) {
        fe = dh_launch_forward_i8(fp, o.stream);
        if (fe == cudaSuccess) { o.lastForwardKernel = 4; return fe; }
        if (fe != cudaErrorNotSupported || mode == 4) return fe;
        cudaGetLastError();
    }
    if (mode == 0 || mode == 3) {
        fe = dh_launch_forward_tma(fp, o.stream);
        if (fe == cudaSuccess) { o.lastForwardKernel = 3; return fe; }
        if (fe != cudaErrorNotSupported || mode == 3) return fe;
        cudaGetLastError();
    }
    if (mode == 0 || mode == 2) {
        fe = dh_launch_forward_reg(fp, o.stream);
        if (fe == cudaSuccess) { o.lastForwardKernel = 2; return fe; }
        if (fe != cudaErrorNotSupported || mode == 2) return fe;
        cudaGetLastError();
    }
    // windows of 256 pixels and more, and IFFT windows whose sides are not
    // powers of two: through the full planes (the plane buffer of the
    // Fourier-plane requests, batch-sized)
    if ((mode == 0 && ((1 << fp.logW) >= 256 || !isPow2(fp.w) || !isPow2(fp.h))) || mode == 5) {
        const size_t Nx = (size_t)(1 << fp.logW) / 2 + 1;
        const size_t frames = (size_t)std::max(o.batchCount * std::max(1, o.avgCount), fp.frameOffset + fp.frameCount);
        const size_t need = frames * o.polCount * (1 << fp.logH) * Nx * sizeof(float2);
        if (o.dFourier.bytes < need && !mayAlloc) return cudaErrorMemoryAllocation;
        fe = o.dFourier.ensure(need);
        if (fe != cudaSuccess) return fe;
        DhFourierParams q;
        memset(&q, 0, sizeof(q));
        q.f = fp;
        q.plane = o.dFourier.as<float2>() + (size_t)fp.frameOffset * o.polCount * (1 << fp.logH) * Nx;
        fe = dh_launch_forward_plane(q, o.stream);
        if (fe == cudaSuccess) { o.lastForwardKernel = 5; return fe; }
        if (fe != cudaErrorNotSupported || mode == 5) return fe;
        cudaGetLastError();
    }
    fe = dh_launch_forward(fp, o.stream);
    if (fe == cudaSuccess) o.lastForwardKernel = 1;
    return fe;
}

// Full-resolution fields by bands of 64 rows (any field size); its scratch
// grows here unless the caller may not allocate.
static cudaError_t launchBands(Object& o, const DhInvParams& ip, bool mayAlloc) {
    if (ip.maxMG > 32 && ip.coefs) {
        // more mode groups than the band kernels' overlap tiles hold: the
        // fields first, then the chunked FP32 overlap of the int16 fields
        DhInvParams fi = ip;
        fi.maxMG = 0;
        fi.modeCount = 0;
        fi.coefs = nullptr;
        cudaError_t e = launchBands(o, fi, mayAlloc);
        if (e != cudaSuccess) return e;
        e = dh_launch_overlap_f32_chunked(ip, o.geo.nx, o.geo.ny, o.stream);
        if (e == cudaSuccess) o.lastOverlapKernel = 1;
        return e;
    }
    // 512-wide fields with IFFT windows up to 64 x 64: 64-point sub-transforms
    // and the exact integer overlap (dh_band64.cu)
    const size_t need64 = dh_field_band64_scratch_bytes(ip, o.overlapKernel);
    if (need64 > 0) {
        if (o.dBigScratch.bytes < need64) {
            if (!mayAlloc) return cudaErrorMemoryAllocation;
            cudaError_t e = o.dBigScratch.ensure(need64);
            if (e != cudaSuccess) return e;
        }
        int used = 0;
        cudaError_t e = dh_launch_field_band64(ip, o.overlapKernel, o.dBigScratch.ptr, o.dBigScratch.bytes, &used, o.stream);
        if (e == cudaSuccess) {
            o.lastInverseKernel = 7;
            o.lastOverlapKernel = used;
            return e;
        }
        if (e != cudaErrorNotSupported) return e;
        cudaGetLastError();
    }
    const size_t need = dh_field_big_scratch_bytes(ip, o.overlapKernel);
    if (need == 0) return cudaErrorNotSupported;
    if (o.dBigScratch.bytes < need) {
        if (!mayAlloc) return cudaErrorMemoryAllocation;
        cudaError_t e = o.dBigScratch.ensure(need);
        if (e != cudaSuccess) return e;
    }
    int used = 0;
    cudaError_t e = dh_launch_field_big(ip, o.overlapKernel, o.dBigScratch.ptr, o.dBigScratch.bytes, &used, o.stream);
    if (e == cudaSuccess) {
        o.lastInverseKernel = 4;
        o.lastOverlapKernel = used;
    }
    return e;
}

// Low-resolution fields of the DFT kernel: its planes in shared memory where
// they fit, else in global scratch (which grows here unless the caller may
// not allocate).
static cudaError_t launchDft(Object& o, const DhInvParams& ip, bool mayAlloc) {
    cudaError_t e = dh_launch_inverse_dft(ip, o.stream);
    if (e != cudaErrorNotSupported) return e;
    cudaGetLastError();
    const size_t need = dh_inverse_dft_global_bytes(ip);
    if (need == 0) return cudaErrorNotSupported;
    if (o.dBigScratch.bytes < need) {
        if (!mayAlloc) return cudaErrorMemoryAllocation;
        e = o.dBigScratch.ensure(need);
        if (e != cudaSuccess) return e;
    }
    return dh_launch_inverse_dft_global(ip, o.dBigScratch.ptr, o.dBigScratch.bytes, o.stream);
}

// Inverse stage: the warp-per-unit kernels for 16/32-pixel low-resolution
// fields; for full-resolution fields the pruned field kernel (fields up to
// 128 x 128) followed by the overlap kernel, else the band kernels; else the
// block-per-unit kernel; low-resolution fields whose sides are not powers of
// two: the DFT kernel.
static cudaError_t launchInverse(Object& o, const DhInvParams& ip, bool mayAlloc = true) {
    if (ip.refCal) {
        // the calibration multiplies the IFFT output in the block-per-unit
        // kernels, or for larger full-resolution fields in k_field_big
        cudaError_t e = dh_launch_inverse(ip, o.stream);
        if (e == cudaSuccess) { o.lastInverseKernel = 1; o.lastOverlapKernel = 1; return e; }
        if (e != cudaErrorNotSupported) return e;
        cudaGetLastError();
        if (!ip.lowres) return launchBands(o, ip, mayAlloc);   // k_field_big: fields beyond one block
        e = launchDft(o, ip, mayAlloc);
        if (e == cudaSuccess) { o.lastInverseKernel = 6; o.lastOverlapKernel = 1; }
        return e;
    }
    if (o.inverseKernel == 2) return launchBands(o, ip, mayAlloc);
    if (o.inverseKernel == 0 || o.inverseKernel == 3) {   // 3: as 0 where not fused
        cudaError_t e = dh_launch_inverse_lo(ip, o.stream);
        if (e == cudaSuccess) { o.lastInverseKernel = 2; o.lastOverlapKernel = 1; return e; }
        if (e != cudaErrorNotSupported) return e;
        cudaGetLastError();
        // full resolution: field kernel, then the overlap kernel
        int fused = 0;
        e = dh_launch_field_full(ip, o.overlapKernel == 0, &fused, o.stream);
        if (e == cudaSuccess && fused) { o.lastInverseKernel = 3; o.lastOverlapKernel = 2; return e; }
        if (e == cudaErrorNotSupported && fused) {
            cudaGetLastError();
            e = dh_launch_field_full(ip, 0, &fused, o.stream);
        }
        if (e == cudaSuccess) {
            const int nx = 1 << ip.logW, ny = 1 << ip.logH;
            e = dh_launch_overlap_f32(ip, nx, ny, o.stream);
            if (e == cudaErrorNotSupported) {   // beyond its register tiles
                cudaGetLastError();
                e = dh_launch_overlap_f32_chunked(ip, nx, ny, o.stream);
            }
            if (e == cudaSuccess) { o.lastInverseKernel = 3; o.lastOverlapKernel = 1; return e; }
            if (e != cudaErrorNotSupported) return e;
            cudaGetLastError();
            // overlap shape not covered: rerun the whole stage with another kernel
        } else if (e != cudaErrorNotSupported) {
            return e;
        } else {
            cudaGetLastError();
        }
        if (!ip.lowres && ((1 << ip.logW) > 128 || (1 << ip.logH) > 128 || !isPow2(ip.w) || !isPow2(ip.h))) {
            e = launchBands(o, ip, mayAlloc);
            if (e != cudaErrorNotSupported) return e;
            cudaGetLastError();
        }
    }
    cudaError_t e = dh_launch_inverse(ip, o.stream);
    if (e == cudaSuccess) { o.lastInverseKernel = 1; o.lastOverlapKernel = 1; return e; }
    if (e != cudaErrorNotSupported || !ip.lowres) return e;
    // low-resolution fields whose sides are not powers of two
    cudaGetLastError();
    e = launchDft(o, ip, mayAlloc);
    if (e == cudaSuccess) { o.lastInverseKernel = 6; o.lastOverlapKernel = 1; }
    return e;
}

// Reads the kernels' failure flag after the stream has been synchronised.
int objCheckStatus(Object& o) {
    if (o.hStatus && *(volatile int*)o.hStatus) {
        *(volatile int*)o.hStatus = 0;
        return fail(o, ERR_ERROR, "kernel: a completion wait (TMA or tensor-core commit) expired");
    }
    return ERR_SUCCESS;
}

static int launchChunk(Object& o, const DhFwdParams& fp0, const DhInvParams& ip0, int f0, int f1) {
    const Geometry& g = o.geo;
    const int P = o.polCount;
    DhFwdParams fp = fp0;
    const size_t es = o.framesU16 ? 2 : 4;
    fp.frames = static_cast<const char*>(fp0.frames) + (size_t)f0 * fp0.frameStride * es;
    fp.frameCount = f1 - f0;
    fp.frameOffset = f0;
    fp.window = fp0.window + (size_t)f0 * P * g.w * g.h;
    const int timed = o.timing && fp.frameOffset == 0 && f1 == o.batchCount;
    cudaEvent_t* ev = nullptr;
    if (timed) {
        if ((int)o.evStage.size() < 3 * (o.evStageUsed + 1)) {
            for (int i = 0; i < 3; i++) {
                cudaEvent_t e;
                DH_CUDA(o, cudaEventCreate(&e));
                o.evStage.push_back(e);
            }
        }
        ev = &o.evStage[3 * o.evStageUsed];
        o.evStageUsed++;
        DH_CUDA(o, cudaEventRecord(ev[0], o.stream));
    }
    DhInvParams ip = ip0;
    if (ip0.fieldR) {
        const size_t npix = (size_t)g.nx * g.ny;
        ip.window = ip0.window + (size_t)f0 * P * g.w * g.h;
        ip.frameCount = f1 - f0;
        ip.fieldR = ip0.fieldR + (size_t)f0 * P * npix;
        ip.fieldI = ip0.fieldI + (size_t)f0 * P * npix;
        if (ip.field32) ip.field32 = ip0.field32 + (size_t)f0 * P * npix;
        ip.stats = ip0.stats + f0;
        if (ip.coefs) ip.coefs = ip0.coefs + (size_t)f0 * P * o.modeCount;
        // both stages in one launch, on request (inverse choice 3): the
        // tensor-core forward with 16 x 16 low-resolution fields.  Measured
        // slower than the two launches, whose inverse kernel runs many more
        // units at once than the forward kernel's epilogue groups can.
        if ((o.forwardKernel == 0 || o.forwardKernel == 4) && o.inverseKernel == 3 && !ip.refCal) {
            cudaError_t fe = dh_launch_forward_i8_fused(fp, ip, o.stream);
            if (fe == cudaSuccess) {
                o.lastForwardKernel = 4;
                o.lastInverseKernel = 5;
                o.lastOverlapKernel = 1;
                if (timed) {
                    DH_CUDA(o, cudaEventRecord(ev[1], o.stream));
                    DH_CUDA(o, cudaEventRecord(ev[2], o.stream));
                }
                return ERR_SUCCESS;
            }
            if (fe != cudaErrorNotSupported) return failCuda(o, fe, "fused forward/inverse kernel launch");
            cudaGetLastError();
        }
    }
    cudaError_t fe = launchForward(o, fp);
    if (fe != cudaSuccess) return failCuda(o, fe, "forward kernel launch");
    if (timed) DH_CUDA(o, cudaEventRecord(ev[1], o.stream));
    if (ip0.fieldR) DH_CUDA(o, launchInverse(o, ip));
    if (timed) DH_CUDA(o, cudaEventRecord(ev[2], o.stream));
    return ERR_SUCCESS;
}

// Frame averaging (avgCount > 1; digHoloSetBatchAvg, digHolo.cpp:8636-8672):
// the forward stage over all batch x avg frames into a scratch window
// buffer, the phase-aligned average of each batch item's windows into the
// window buffer (k_average_windows, with the batch calibration), then the
// inverse stage over the batch.  The frames must already be staged (fp0).
static int launchAveraged(Object& o, const DhFwdParams& fp0, const DhInvParams& ip) {
    const Geometry& g = o.geo;
    const int B = o.batchCount, A = o.avgCount, P = o.polCount;
    const size_t n = (size_t)g.w * g.h;
    DH_CUDA(o, o.dWindowAvg.ensure((size_t)B * A * P * n * sizeof(float2)));
    DhFwdParams fp = fp0;
    fp.frameCount = B * A;
    fp.frameOffset = 0;
    fp.window = o.dWindowAvg.as<float2>();
    fp.batchCal = nullptr;   // per batch item, after the average
    fp.batchCalCount = 0;
    cudaEvent_t* ev = nullptr;
    if (o.timing) {
        if ((int)o.evStage.size() < 3 * (o.evStageUsed + 1)) {
            for (int i = 0; i < 3; i++) {
                cudaEvent_t e;
                DH_CUDA(o, cudaEventCreate(&e));
                o.evStage.push_back(e);
            }
        }
        ev = &o.evStage[3 * o.evStageUsed];
        o.evStageUsed++;
        DH_CUDA(o, cudaEventRecord(ev[0], o.stream));
    }
    cudaError_t fe = launchForward(o, fp);
    if (fe != cudaSuccess) return failCuda(o, fe, "forward kernel launch");
    DH_CUDA(o, dh_launch_average_windows(fp.window, fp0.window, B, A, o.cfg.avgMode, P, (int)n, fp0.batchCal,
                                         fp0.batchCalCount, o.stream));
    if (ev) DH_CUDA(o, cudaEventRecord(ev[1], o.stream));
    if (ip.fieldR) DH_CUDA(o, launchInverse(o, ip));
    if (ev) DH_CUDA(o, cudaEventRecord(ev[2], o.stream));
    return ERR_SUCCESS;
}

// Sums the forward / inverse kernel times of the batches timed since the
// last call: out = {forward ms, inverse ms, batch count}; then resets.
int objStageTimes(Object& o, float* out) {
    out[0] = out[1] = out[2] = 0.f;
    if (o.evStageUsed == 0) return ERR_SUCCESS;
    DH_CUDA(o, cudaEventSynchronize(o.evStage[3 * o.evStageUsed - 1]));
    for (int i = 0; i < o.evStageUsed; i++) {
        float a = 0.f, b = 0.f;
        DH_CUDA(o, cudaEventElapsedTime(&a, o.evStage[3 * i], o.evStage[3 * i + 1]));
        DH_CUDA(o, cudaEventElapsedTime(&b, o.evStage[3 * i + 1], o.evStage[3 * i + 2]));
        out[0] += a;
        out[1] += b;
    }
    out[2] = (float)o.evStageUsed;
    o.evStageUsed = 0;
    return ERR_SUCCESS;
}

// HG -> LG transform of G mode groups, T[i * M + j] (HG mode i, LG mode j),
// block-diagonal by group (digHoloLGInit, digHolo.cpp:9909-10040, with the
// weights of digHoloLGtoHGcoef, digHolo.cpp:9819-9907: the Beijersbergen
// mode-converter expansion).  Group g holds HG (g - c, c) at position c and
// LG l = g - 2r, p = (g - |l|) / 2 at position r; with (n, m) = (p, p - l)
// for l < 0, else (l + p, p), the weight of HG (hm, hn) is
// [t^hm] (1 + t)^n (1 - t)^m * sqrt(hm! hn! / (n! m! 2^g)) * i^(g + hm),
// negated for odd g and l > 0; FP64, rounded once to complex64.
static void lgTransform(int G, std::vector<float2>& T) {
    const int M = G * (G + 1) / 2;
    T.assign((size_t)M * M, make_float2(0.f, 0.f));
    std::vector<double> poly, lf(2 * G + 2, 0.0);
    for (int k = 1; k < (int)lf.size(); k++) lf[k] = lf[k - 1] + std::log((double)k);   // log k!
    int base = 0;
    for (int g = 0; g < G; g++) {
        for (int r = 0; r <= g; r++) {
            const int l = g - 2 * r, p = (g - std::abs(l)) / 2;
            const int n = l < 0 ? p : l + p, m = l < 0 ? p - l : p;
            // (1 + t)^n (1 - t)^m, exact in double for the group sizes here
            poly.assign(1, 1.0);
            for (int k = 0; k < n + m; k++) {
                const double sgn = k < n ? 1.0 : -1.0;
                poly.push_back(0.0);
                for (int e = (int)poly.size() - 1; e >= 1; e--) poly[e] += sgn * poly[e - 1];
            }
            for (int c = 0; c <= g; c++) {
                const int hm = g - c, hn = c;
                const double puv = hm < (int)poly.size() ? poly[hm] : 0.0;
                double v = puv * std::exp(0.5 * (lf[hm] + lf[hn] - lf[n] - lf[m]) - 0.5 * g * std::log(2.0));
                if ((g & 1) && l > 0) v = -v;
                const int q = (g + hm) & 3;   // i^q
                const float2 w = q == 0 ? make_float2((float)v, 0.f)
                                 : q == 1 ? make_float2(0.f, (float)v)
                                 : q == 2 ? make_float2((float)-v, 0.f)
                                          : make_float2(0.f, (float)-v);
                T[(size_t)(base + c) * M + (base + r)] = w;
            }
        }
        base += g + 1;
    }
}

const float2* objOutputCoefs(const Object& o) {
    return o.basisActive ? o.dCoefsOut.as<float2>() : o.dCoefs.as<float2>();
}
int objOutputModes(const Object& o) { return o.basisActive ? o.modeCountOut : o.modeCount; }

// The coefficients in the configured basis (digHoloApplyBasisTransform,
// digHolo.cpp:9469-9600): HG for type 0, an unknown type or an invalid
// custom matrix; LG (type 1) over all modes; custom (type 2): the leading
// min(M, in) x min(M, out) block of the [in][out] matrix, min(M, out) modes
// out.  The device matrix is rebuilt when the type, the mode count or the
// custom matrix changes (after the stream has drained: a batch in flight may
// still read the previous one).
static int applyBasis(Object& o) {
    const int M = o.modeCount;
    int t = o.cfg.basisType;
    if (t < 0 || t > 2 || (t == 2 && (o.basisCustom.empty() || o.basisCustomIn <= 0 || o.basisCustomOut <= 0))) t = 0;
    o.basisActive = 0;
    o.modeCountOut = M;
    if (t == 0 || M <= 0 || !o.dCoefs.ptr) return ERR_SUCCESS;
    const int din = t == 1 ? M : std::min(M, o.basisCustomIn);
    const int dout = t == 1 ? M : std::min(M, o.basisCustomOut);
    if (o.basisTType != t || o.basisTModes != M || (t == 2 && o.basisTVersion != o.basisCustomVersion)) {
        std::vector<float2> T;
        if (t == 1) {
            int G = 0;
            while ((G + 1) * (G + 2) / 2 <= M) G++;
            lgTransform(G, T);
        } else {
            T.resize((size_t)din * dout);
            const float* full = o.basisCustom.data();
            for (int i = 0; i < din; i++)
                for (int j = 0; j < dout; j++) {
                    const size_t src = 2 * ((size_t)i * o.basisCustomOut + j);
                    T[(size_t)i * dout + j] = make_float2(full[src], full[src + 1]);
                }
        }
        DH_CUDA(o, cudaStreamSynchronize(o.stream));
        DH_CUDA(o, o.dBasisT.ensure(T.size() * sizeof(float2)));
        DH_CUDA(o, cudaMemcpy(o.dBasisT.ptr, T.data(), T.size() * sizeof(float2), cudaMemcpyHostToDevice));
        o.basisTType = t;
        o.basisTModes = M;
        o.basisTVersion = o.basisCustomVersion;
    }
    const int rows = o.batchCount * o.polCount;
    DH_CUDA(o, o.dCoefsOut.ensure((size_t)rows * dout * sizeof(float2)));
    DH_CUDA(o, dh_launch_basis_transform(o.dCoefs.as<float2>(), o.dCoefsOut.as<float2>(), o.dBasisT.as<float2>(), rows,
                                         M, din, dout, o.stream));
    o.basisActive = t;
    o.basisDimIn = din;
    o.modeCountOut = dout;
    return ERR_SUCCESS;
}

// Releases the captured batch graphs of the object.
void objReleaseGraphs(Object& o) {
    for (auto& g : o.graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    o.graphs.clear();
    o.graphPending.clear();
}

// Device-resident frames: the batch's forward and inverse launches replayed
// from a CUDA graph (one cudaGraphLaunch instead of the launch sequence and
// its host-side checks).  The key holds every argument of those launches
// (both parameter blocks, the kernel choices, the batch size and the device
// allocation generation), so a graph is replayed only for launches identical
// to the ones it captured.  Launches run directly the first time their
// arguments other than the frame pointer are seen (kernel attributes, tensor
// maps and scratch buffers are settled then); after that every new frame
// buffer is captured on first use (a ring of acquisition buffers gets one
// graph each).  At most eight graphs and eight settled argument sets are kept.
static int launchBatchDevice(Object& o, const DhFwdParams& fp, const DhInvParams& ip) {
    const int B = o.batchCount;
    // the default streams cannot be captured; a stream the caller is
    // capturing already records the launches into the caller's graph
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool defaultStream = o.stream == nullptr || o.stream == cudaStreamLegacy || o.stream == cudaStreamPerThread;
    if (!o.useGraphs || o.timing || defaultStream || cudaStreamIsCapturing(o.stream, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return launchChunk(o, fp, ip, 0, B);
    }
    const int choice[4] = {o.forwardKernel, o.inverseKernel, o.overlapKernel, B};
    const unsigned long long gen = devBufGeneration();
    std::vector<unsigned char> key(sizeof(fp) + sizeof(ip) + sizeof(choice) + sizeof(gen));
    unsigned char* k = key.data();
    memcpy(k, &fp, sizeof(fp));
    memcpy(k + sizeof(fp), &ip, sizeof(ip));
    memcpy(k + sizeof(fp) + sizeof(ip), choice, sizeof(choice));
    memcpy(k + sizeof(fp) + sizeof(ip) + sizeof(choice), &gen, sizeof(gen));
    for (auto& g : o.graphs) {
        if (g.key != key) continue;
        DH_CUDA(o, cudaGraphLaunch(g.exec, o.stream));
        o.lastForwardKernel = g.fwdKernel;
        o.lastInverseKernel = g.invKernel;
        o.lastOverlapKernel = g.ovlKernel;
        return ERR_SUCCESS;
    }
    // the same launches on other frames have run directly before: capture now
    std::vector<unsigned char> shape = key;
    memset(shape.data() + offsetof(DhFwdParams, frames), 0, sizeof(fp.frames));
    if (std::find(o.graphPending.begin(), o.graphPending.end(), shape) == o.graphPending.end()) {
        if (o.graphPending.size() >= 8) o.graphPending.erase(o.graphPending.begin());
        o.graphPending.push_back(std::move(shape));
        return launchChunk(o, fp, ip, 0, B);
    }
    if (cudaStreamBeginCapture(o.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        if (++o.graphFailures >= 3) o.useGraphs = 0;
        return launchChunk(o, fp, ip, 0, B);
    }
    const int r = launchChunk(o, fp, ip, 0, B);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(o.stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (r == ERR_SUCCESS && e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (r != ERR_SUCCESS || e != cudaSuccess || !exec) {
        // nothing of the capture ran: launch directly; give up on graphs
        // after repeated failures
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        if (++o.graphFailures >= 3) o.useGraphs = 0;
        return launchChunk(o, fp, ip, 0, B);
    }
    if (o.graphs.size() >= 8) {
        cudaGraphExecDestroy(o.graphs.front().exec);
        o.graphs.erase(o.graphs.begin());
    }
    Object::BatchGraph g;
    g.key = std::move(key);
    g.exec = exec;
    g.fwdKernel = o.lastForwardKernel;
    g.invKernel = o.lastInverseKernel;
    g.ovlKernel = o.lastOverlapKernel;
    o.graphs.push_back(std::move(g));
    DH_CUDA(o, cudaGraphLaunch(exec, o.stream));
    return ERR_SUCCESS;
}

// Full pipeline for the batch: stage -> forward -> inverse (+overlap).
// With host frames the batch is split in two chunks: the kernels of the
// first run while the second's window copies arrive, so only the small
// second chunk's kernels follow the last copy.  Each copy operation costs a
// few microseconds of DMA setup, so more chunks lengthen the copy.
static int processBatchLocked(Object& o, int syncCoefs);

// Transposed uint16 frames (digHoloSetBatchUint16 with transpose): each frame
// is stored with x and y swapped (frameWidth rows of frameHeight pixels); it
// is transposed on the device (k_untranspose_u16), then processed like any
// device batch.  This is the documented intent of the reference's transposing
// converter (convert_int16tofloat32, digHolo.cpp:1206-1229), whose lane
// permutation scrambles every other output row.
// digHoloWavelengthUpdate (digHolo.cpp:7823-7862): a pending array replaces
// the one in use; with none, the centre wavelength alone; an array of one
// wavelength is replaced by the centre wavelength.
void objWavelengthUpdate(Object& o) {
    if (!o.wavelengthsValid && !o.wavelengthsNew.empty()) {
        o.wavelengths = o.wavelengthsNew;
        o.wavelengthsValid = 1;
    } else if (o.wavelengths.empty()) {
        o.wavelengths.assign(1, o.cfg.wavelengthCentre);
        o.wavelengthsValid = 1;
    }
    if (o.wavelengths.size() == 1) o.wavelengths[0] = o.cfg.wavelengthCentre;
}

// A batch of frames at L > 1 wavelengths (digHoloProcessBatchFrequencySweep*,
// digHolo.cpp:5046-5080; digHoloIFFTRoutine's per-frame wavenumber,
// digHolo.cpp:8641-8700; one reference wave per wavelength,
// digHolo.cpp:10386-10504).  Frame i belongs to wavelength i mod L
// (wavelength the fast axis of the input) or i / (B / L) (slow axis), and
// output o of that frame is sub L + lambda (fast) or lambda (B / L) + sub
// (slow) (WavelengthOrderingCalc, digHolo.cpp:2656-2700).  The frames of
// each wavelength go through the batch path as one sub-batch: the IFFT
// window spans the first and last wavelength (digHolo.cpp:7868-8048), the
// Fourier-window mask, its centre and the reference wave follow the
// sub-batch's wavelength; the outputs are scattered to their positions.
// The batch count must be a multiple of L; frame averaging is not combined
// with it here.
static int processSweepLocked(Object& o, int syncCoefs) {
    int r = objInitDevice(o);
    if (r) return r;
    const std::vector<float> lams = o.wavelengths;
    const int L = (int)lams.size();
    const Config saved = o.cfg;
    const int B = std::max(1, saved.batchCount);
    if (!o.frames) return fail(o, ERR_NULLPOINTER, "frame buffer not set");
    if (B % L)
        return fail(o, ERR_INVALIDDIMENSION, "multi-wavelength batches: the batch count must be a multiple of the wavelength count");
    const int S = B / L;
    const bool inFast = saved.wavelengthOrdering[0] == 0, outFast = saved.wavelengthOrdering[1] == 0;
    const size_t es = o.framesU16 ? 2 : 4;
    const size_t frameBytes = (size_t)saved.frameWidth * saved.frameHeight * es;
    const void* framesIn = o.frames;
    const int onDevice = isDevicePointer(framesIn);
    const std::vector<float> calSaved = o.batchCal;
    const int calEnabled = o.batchCalEnabled, calCount = o.batchCalCount, calPol = o.batchCalPolCount;
    struct Restore {
        Object& o; Config c; const void* f; int d, t; std::vector<float> cal; int calCount;
        ~Restore() {
            o.cfg = c; o.frames = f; o.framesOnDevice = d; o.framesTransposed = t;
            o.batchCal = cal; o.batchCalCount = calCount; o.batchCalVersion++;
            o.sweepLambda = -1; o.batchCalCaller = nullptr;
        }
    } restore{o, saved, o.frames, o.framesOnDevice, o.framesTransposed, calSaved, calCount};
    // the reference-wave calibration of each sub-batch: its wavelength index,
    // the batch's centre wavelength and the caller's batch calibration
    o.sweepCentre = saved.wavelengthCentre;
    o.batchCalCaller = &restore.cal;
    o.batchCalCallerCount = calCount;
    o.batchCalCallerPol = calPol;
    // frame averaging: each item's A frames, gathered per sub-batch in the
    // sequential order (item j's k-th frame at j A + k); the reference's
    // frame of input item b and average k (digHolo.cpp:8661-8672): b A + k
    // (sequential), k B + b (interlaced), b + k L (sweeps)
    const int A = std::max(1, saved.avgCount);
    const int avgMode = saved.avgMode;
    DH_CUDA(o, o.dSweepFrames.ensure((size_t)S * A * frameBytes));
    int P = 0, M = 0, Mout = 0, nx = 0, ny = 0, keep32 = o.keepField32, active = 0;
    for (int l = 0; l < L; l++) {
        const size_t in0 = inFast ? (size_t)l : (size_t)l * S, inStep = inFast ? (size_t)L : 1;
        for (int k = 0; k < A; k++) {
            size_t first = in0, stride = inStep;   // in frames
            if (A > 1) {
                if (avgMode == 0) { first = in0 * A + k; stride = inStep * A; }
                else if (avgMode == 1) first = (size_t)k * B + in0;
                else first = in0 + (size_t)k * L;
            }
            const char* src = static_cast<const char*>(framesIn) + first * frameBytes;
            DH_CUDA(o, cudaMemcpy2DAsync(static_cast<char*>(o.dSweepFrames.ptr) + (size_t)k * frameBytes,
                                         (size_t)A * frameBytes, src, stride * frameBytes, frameBytes, S,
                                         onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, o.stream));
        }
        if (calEnabled && calCount > 0) {
            // the batch calibration of each frame's input index
            std::vector<float> c((size_t)calPol * S * 2);
            for (int p = 0; p < calPol; p++)
                for (int j = 0; j < S; j++) {
                    const int in = inFast ? l + L * j : l * S + j;
                    const size_t srcIdx = ((size_t)p * calCount + (in % calCount)) * 2;
                    c[((size_t)p * S + j) * 2] = calSaved[srcIdx];
                    c[((size_t)p * S + j) * 2 + 1] = calSaved[srcIdx + 1];
                }
            o.batchCal = c;
            o.batchCalCount = S;
            o.batchCalVersion++;
        }
        o.frames = o.dSweepFrames.ptr;
        o.framesOnDevice = 1;
        o.framesTransposed = 0;
        o.cfg = saved;
        o.cfg.batchCount = S;
        o.cfg.avgMode = 0;   // gathered in the sequential order above
        o.cfg.wavelengthCentre = lams[l];
        o.cfg.lambdaRange[0] = lams[0];
        o.cfg.lambdaRange[1] = lams[L - 1];
        o.sweepLambda = l;
        r = processBatchLocked(o, 0);
        if (r) return r;
        P = o.polCount; M = o.modeCount; nx = o.geo.nx; ny = o.geo.ny;
        active = o.basisActive; Mout = o.modeCountOut;
        if (l == 0) {
            DH_CUDA(o, o.dAccCoefs.ensure((size_t)B * P * std::max(1, M) * sizeof(float2)));
            DH_CUDA(o, o.dAccCoefsOut.ensure((size_t)B * P * std::max(1, Mout) * sizeof(float2)));
            DH_CUDA(o, o.dAccFieldR.ensure((size_t)B * P * nx * ny * sizeof(short)));
            DH_CUDA(o, o.dAccFieldI.ensure((size_t)B * P * nx * ny * sizeof(short)));
            if (keep32) DH_CUDA(o, o.dAccField32.ensure((size_t)B * P * nx * ny * sizeof(float2)));
            DH_CUDA(o, o.dAccStats.ensure((size_t)ANALYSIS_COUNT * P * (B + 1) * sizeof(float)));
        }
        // rows of this sub-batch to their output positions
        auto scatter = [&](void* dst, const void* srcRows, size_t rowBytes) -> cudaError_t {
            char* d = static_cast<char*>(dst) + (size_t)(outFast ? l : l * S) * rowBytes;
            return cudaMemcpy2DAsync(d, outFast ? (size_t)L * rowBytes : rowBytes, srcRows, rowBytes, rowBytes, S,
                                     cudaMemcpyDeviceToDevice, o.stream);
        };
        if (M > 0) DH_CUDA(o, scatter(o.dAccCoefs.ptr, o.dCoefs.ptr, (size_t)P * M * sizeof(float2)));
        if (active && Mout > 0) DH_CUDA(o, scatter(o.dAccCoefsOut.ptr, o.dCoefsOut.ptr, (size_t)P * Mout * sizeof(float2)));
        DH_CUDA(o, scatter(o.dAccFieldR.ptr, o.dFieldR.ptr, (size_t)P * nx * ny * sizeof(short)));
        DH_CUDA(o, scatter(o.dAccFieldI.ptr, o.dFieldI.ptr, (size_t)P * nx * ny * sizeof(short)));
        if (keep32) DH_CUDA(o, scatter(o.dAccField32.ptr, o.dField32.ptr, (size_t)P * nx * ny * sizeof(float2)));
        // statistics [param][pol][S + 1] -> [param][pol][B + 1]
        const int rowsStat = ANALYSIS_COUNT * P;
        float* accS = o.dAccStats.as<float>();
        const float* subS = o.dStats.as<float>();
        if (!outFast) {
            DH_CUDA(o, cudaMemcpy2DAsync(accS + (size_t)l * S, (size_t)(B + 1) * 4, subS, (size_t)(S + 1) * 4, (size_t)S * 4,
                                         rowsStat, cudaMemcpyDeviceToDevice, o.stream));
        } else {
            for (int q = 0; q < rowsStat; q++)
                DH_CUDA(o, cudaMemcpy2DAsync(accS + (size_t)q * (B + 1) + l, (size_t)L * 4, subS + (size_t)q * (S + 1), 4, 4, S,
                                             cudaMemcpyDeviceToDevice, o.stream));
        }
    }
    // the whole batch's outputs in the handle's buffers
    o.batchCount = B;
    const size_t nf = (size_t)B * P * nx * ny;
    if (M > 0) {
        DH_CUDA(o, o.dCoefs.ensure((size_t)B * P * M * sizeof(float2)));
        DH_CUDA(o, cudaMemcpyAsync(o.dCoefs.ptr, o.dAccCoefs.ptr, (size_t)B * P * M * sizeof(float2), cudaMemcpyDeviceToDevice, o.stream));
    }
    if (active && Mout > 0) {
        DH_CUDA(o, o.dCoefsOut.ensure((size_t)B * P * Mout * sizeof(float2)));
        DH_CUDA(o, cudaMemcpyAsync(o.dCoefsOut.ptr, o.dAccCoefsOut.ptr, (size_t)B * P * Mout * sizeof(float2), cudaMemcpyDeviceToDevice, o.stream));
    }
    DH_CUDA(o, o.dFieldR.ensure(nf * sizeof(short)));
    DH_CUDA(o, o.dFieldI.ensure(nf * sizeof(short)));
    DH_CUDA(o, cudaMemcpyAsync(o.dFieldR.ptr, o.dAccFieldR.ptr, nf * sizeof(short), cudaMemcpyDeviceToDevice, o.stream));
    DH_CUDA(o, cudaMemcpyAsync(o.dFieldI.ptr, o.dAccFieldI.ptr, nf * sizeof(short), cudaMemcpyDeviceToDevice, o.stream));
    if (keep32) {
        DH_CUDA(o, o.dField32.ensure(nf * sizeof(float2)));
        DH_CUDA(o, cudaMemcpyAsync(o.dField32.ptr, o.dAccField32.ptr, nf * sizeof(float2), cudaMemcpyDeviceToDevice, o.stream));
    }
    DH_CUDA(o, o.dStats.ensure((size_t)ANALYSIS_COUNT * P * (B + 1) * sizeof(float)));
    DH_CUDA(o, cudaMemcpyAsync(o.dStats.ptr, o.dAccStats.ptr, (size_t)ANALYSIS_COUNT * P * (B + 1) * sizeof(float),
                               cudaMemcpyDeviceToDevice, o.stream));
    // the tables of the last sub-batch's wavelength are not the configuration's
    o.preparedValid = 0;
    o.lastFwdValid = 0;
    o.fourierValid = 0;
    o.metricsValid = 0;
    if (syncCoefs) return objCoefsToHost(o);
    return ERR_SUCCESS;
}

static int processAnyLocked(Object& o, int syncCoefs) {
    objWavelengthUpdate(o);
    if (o.wavelengths.size() > 1) return processSweepLocked(o, syncCoefs);
    o.cfg.lambdaRange[0] = o.cfg.lambdaRange[1] = 0.f;
    return processBatchLocked(o, syncCoefs);
}

int objProcessBatch(Object& o, int syncCoefs) {
    std::lock_guard<std::mutex> guard(o.lock);
    if (!(o.framesTransposed && o.framesU16)) return processAnyLocked(o, syncCoefs);
    int r = objInitDevice(o);
    if (r) return r;
    if (!o.frames) return fail(o, ERR_NULLPOINTER, "frame buffer not set");
    const Config& c = o.cfg;
    const int frames = std::max(1, c.batchCount) * std::max(1, c.avgCount);
    const size_t bytes = (size_t)frames * c.frameWidth * c.frameHeight * sizeof(unsigned short);
    const void* src = o.frames;
    if (!isDevicePointer(o.frames)) {
        DH_CUDA(o, o.dTransRaw.ensure(bytes));
        DH_CUDA(o, cudaMemcpyAsync(o.dTransRaw.ptr, o.frames, bytes, cudaMemcpyHostToDevice, o.stream));
        src = o.dTransRaw.ptr;
    }
    DH_CUDA(o, o.dTransFrames.ensure(bytes));
    // input [frameWidth rows][frameHeight columns] -> [frameHeight rows][frameWidth columns]
    DH_CUDA(o, dh_launch_untranspose_u16(static_cast<const unsigned short*>(src), o.dTransFrames.as<unsigned short>(),
                                         c.frameHeight, c.frameWidth, frames, o.stream));
    struct Restore {
        Object& o; const void* f; int d;
        ~Restore() { o.frames = f; o.framesOnDevice = d; o.framesTransposed = 1; }
    } restore{o, o.frames, o.framesOnDevice};
    o.frames = o.dTransFrames.ptr;
    o.framesOnDevice = 1;
    o.framesTransposed = 0;
    return processAnyLocked(o, syncCoefs);
}

// ------------------------------------------------------------------ kernel planner
// The counterpart of the reference's FFTW planning (digHoloConfigSetFFTWPlanMode,
// digHolo.h:1808; FFTW_MEASURE and up time candidate plans, digHolo.cpp:7439-7531,
// and keep them as wisdom, digHolo.cpp:7424-7437): with plan mode 1-3 and
// automatic kernel choices, the first batch of each shape (frame and window
// sizes, polarisations, pixel type, frame source, resolution mode, mode
// groups, batch size rounded up to a power of two up to 512, overlap choice)
// is also run through every forward x inverse kernel pair that supports it,
// each timed with CUDA events on up to 512 of its frames (best of 1, 3 or 5
// runs for MEASURE, PATIENT, EXHAUSTIVE), and the fastest pair is used for
// every later batch of that shape.  The table is process-wide like FFTW's wisdom; with a wisdom file
// named (digHoloFFTWWisdomFilename) it is loaded from it before the first
// lookup and written back after every new entry.

namespace {
struct PlanEntry {
    int fwd, inv;
    float ms;
};
std::mutex gPlanLock;
std::map<std::string, PlanEntry> gPlans;
std::string gPlanFile;
bool gPlanLoaded = true;
int gPlanRuns = 0;
const char* kPlanHeader = "digholo_b200 kernel plans v1";

void planLoadLocked() {
    if (gPlanLoaded) return;
    gPlanLoaded = true;
    std::ifstream f(gPlanFile);
    std::string line;
    if (!f || !std::getline(f, line) || line != kPlanHeader) return;
    while (std::getline(f, line)) {
        const size_t t = line.find('\t');
        if (t == std::string::npos) continue;
        std::istringstream v(line.substr(t + 1));
        PlanEntry e;
        if (v >> e.fwd >> e.inv >> e.ms) gPlans[line.substr(0, t)] = e;
    }
}

void planSaveLocked() {
    if (gPlanFile.empty()) return;
    std::ofstream f(gPlanFile, std::ios::trunc);
    if (!f) return;
    f << kPlanHeader << "\n";
    for (const auto& kv : gPlans) f << kv.first << "\t" << kv.second.fwd << " " << kv.second.inv << " " << kv.second.ms << "\n";
}

std::string planKey(const Object& o) {
    const Geometry& g = o.geo;
    int bucket = 1;   // batch sizes by powers of two up to the planner's 512-frame trials
    while (bucket < o.batchCount && bucket < 512) bucket <<= 1;
    char k[256];
    snprintf(k, sizeof(k), "%d %d %d %d %d %d %d %d %d %d %d %d %d", o.cfg.frameWidth, o.cfg.frameHeight, o.polCount,
             o.framesU16, o.framesOnDevice, g.W, g.H, g.w, g.h, o.cfg.resolutionIdx, o.cfg.maxMG, bucket, o.overlapKernel);
    return k;
}
}  // namespace

int planForget() {
    std::lock_guard<std::mutex> g(gPlanLock);
    gPlans.clear();
    return ERR_SUCCESS;
}
int planFilename(const char* filename) {
    std::lock_guard<std::mutex> g(gPlanLock);
    gPlanFile = filename ? filename : "";
    gPlanLoaded = gPlanFile.empty();
    return ERR_SUCCESS;
}
int planRuns() {
    std::lock_guard<std::mutex> g(gPlanLock);
    return gPlanRuns;
}

// The tuned pair for the handle's current shape (after a batch was prepared): 1 if there is one.
int objPlanLookup(Object& o, int* fwd, int* inv, float* ms) {
    std::lock_guard<std::mutex> g(gPlanLock);
    planLoadLocked();
    auto it = gPlans.find(planKey(o));
    if (it == gPlans.end()) return 0;
    if (fwd) *fwd = it->second.fwd;
    if (inv) *inv = it->second.inv;
    if (ms) *ms = it->second.ms;
    return 1;
}

// Times every forward x inverse pair on (up to 512 frames of) the batch just
// processed (frames as staged for it: fp) and records the fastest; the
// winner then runs once more over the whole batch so that the batch's
// outputs are its.
static int planBatch(Object& o, const DhFwdParams& fp, const DhInvParams& ip) {
    const int B = o.batchCount, BT = std::min(B, 512);
    const int saveF = o.forwardKernel, saveI = o.inverseKernel, saveT = o.timing;
    const std::string saveErr = o.lastError;
    const int reps = o.cfg.fftwPlanMode >= 3 ? 5 : (o.cfg.fftwPlanMode == 2 ? 3 : 1);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DH_CUDA(o, cudaEventCreate(&e0));
    DH_CUDA(o, cudaEventCreate(&e1));
    PlanEntry best{0, 0, FLT_MAX};
    static const int fwds[] = {4, 3, 2, 5, 1};
    static const int invs[] = {0, 1, 2, 3};
    o.timing = 0;
    o.quietErrors = 1;
    for (int f : fwds) {
        for (int i : invs) {
            if (i == 3 && f != 4) continue;                         // fused only with the tensor-core forward
            if (i == 2 && o.cfg.resolutionIdx != 0) continue;       // bands: full resolution
            o.forwardKernel = f;
            o.inverseKernel = i;
            int r = launchChunk(o, fp, ip, 0, BT);
            cudaError_t ce = cudaStreamSynchronize(o.stream);
            if (r || ce != cudaSuccess || objCheckStatus(o)) { cudaGetLastError(); continue; }
            float ms = FLT_MAX;
            for (int k = 0; k < reps && r == 0; k++) {
                cudaEventRecord(e0, o.stream);
                r = launchChunk(o, fp, ip, 0, BT);
                cudaEventRecord(e1, o.stream);
                if (cudaEventSynchronize(e1) != cudaSuccess) r = ERR_ERROR;
                float t = 0.f;
                if (r == 0 && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) ms = std::min(ms, t);
            }
            cudaGetLastError();
            if (r == 0 && ms < best.ms) best = PlanEntry{f, i, ms};
        }
    }
    o.quietErrors = 0;
    o.timing = saveT;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int r = ERR_SUCCESS;
    if (best.ms < FLT_MAX) {
        o.forwardKernel = best.fwd;
        o.inverseKernel = best.inv;
        r = launchChunk(o, fp, ip, 0, B);
        std::lock_guard<std::mutex> g(gPlanLock);
        planLoadLocked();
        gPlans[planKey(o)] = best;
        gPlanRuns++;
        planSaveLocked();
    }
    o.forwardKernel = saveF;
    o.inverseKernel = saveI;
    o.lastError = saveErr;
    return r;
}

static int processBatchLocked(Object& o, int syncCoefs) {
    int r = prepare(o);
    if (r) return r;
    r = updateBasis(o);
    if (r) return r;
    // kernel planner: the tuned kernel pair for this shape, or a tuning run
    // after this batch (plan modes above ESTIMATE, automatic kernel choices)
    struct ChoiceRestore {
        Object& o; int f, i; bool active;
        ~ChoiceRestore() { if (active) { o.forwardKernel = f; o.inverseKernel = i; } }
    } choiceRestore{o, o.forwardKernel, o.inverseKernel, false};
    bool planNeeded = false;
    bool earlyCoefs = false;
    if (o.cfg.fftwPlanMode > 0 && o.forwardKernel == 0 && o.inverseKernel == 0 && o.avgCount <= 1 && !o.useSnaps &&
        !objRefCalApplies(o)) {
        int pf = 0, pi = 0;
        if (objPlanLookup(o, &pf, &pi, nullptr)) {
            o.forwardKernel = pf;
            o.inverseKernel = pi;
            choiceRestore.active = true;
        } else {
            planNeeded = true;
        }
    }
    const Geometry& g = o.geo;
    const int B = o.batchCount, P = o.polCount;
    if (o.modeCount > 0) DH_CUDA(o, o.dCoefs.ensure((size_t)B * P * o.modeCount * sizeof(float2)));
    DhFwdParams fp;
    forwardParams(o, fp);
    DhInvParams ip;
    inverseParams(o, ip, 1);
    r = calParams(o, ip);
    if (r) return r;
    // the last stats column (aggregate over the batch) is filled on request
    if (o.avgCount > 1) {
        r = stageFrames(o, 0, B * o.avgCount, fp, 0);
        if (r) return r;
        r = launchAveraged(o, fp, ip);
        if (r) return r;
    } else if (o.framesOnDevice) {
        r = stageFrames(o, 0, B, fp, 0);
        if (r) return r;
        r = launchBatchDevice(o, fp, ip);
        if (r) return r;
    } else {
        // copies of this call must not overwrite the staging buffer while an
        // earlier call's kernels may still read it
        DH_CUDA(o, cudaEventRecord(o.evStart, o.stream));
        DH_CUDA(o, cudaStreamWaitEvent(o.copyStream, o.evStart, 0));
        if (P > 1) DH_CUDA(o, cudaStreamWaitEvent(o.copyStream2, o.evStart, 0));
        const int tail = B >= 32 ? std::max(1, B / 16) : 0;
        const int bounds[3] = {0, B - tail, B};
        // coefficients of each chunk go to the host as soon as its kernels
        // end (HG output basis: nothing is applied to them after the loop)
        const size_t chunkCoef = (size_t)P * o.modeCount * sizeof(float2);
        earlyCoefs = syncCoefs && o.modeCount > 0 && o.cfg.basisType == 0 && !planNeeded && o.dCoefs.ptr;
        if (earlyCoefs) {
            if (!o.hCoefs.ensure((size_t)B * chunkCoef)) return fail(o, ERR_MEMORYALLOCATION, "host coefficient buffer");
            DH_CUDA(o, cudaStreamWaitEvent(o.d2hStream, o.evStart, 0));
        }
        int slot = 0;
        for (int c = 0; c < 2; c++) {
            const int f0 = bounds[c], f1 = bounds[c + 1];
            if (f1 <= f0) continue;
            DhFwdParams fpc = fp;
            r = stageFrames(o, f0, f1, fpc, 1);
            if (r) return r;
            DH_CUDA(o, cudaEventRecord(o.evCopy[slot], o.copyStream));
            DH_CUDA(o, cudaStreamWaitEvent(o.stream, o.evCopy[slot], 0));
            if (P > 1) {
                DH_CUDA(o, cudaEventRecord(o.evCopy2[slot], o.copyStream2));
                DH_CUDA(o, cudaStreamWaitEvent(o.stream, o.evCopy2[slot], 0));
            }
            r = launchChunk(o, fpc, ip, f0, f1);
            if (r) return r;
            if (earlyCoefs) {
                DH_CUDA(o, cudaEventRecord(o.evChunk[slot], o.stream));
                DH_CUDA(o, cudaStreamWaitEvent(o.d2hStream, o.evChunk[slot], 0));
                DH_CUDA(o, cudaMemcpyAsync(o.hCoefs.as<char>() + (size_t)f0 * chunkCoef,
                                           o.dCoefs.as<char>() + (size_t)f0 * chunkCoef, (size_t)(f1 - f0) * chunkCoef,
                                           cudaMemcpyDeviceToHost, o.d2hStream));
            }
            slot ^= 1;
        }
        if (earlyCoefs) {
            DH_CUDA(o, cudaEventRecord(o.evD2H, o.d2hStream));
            DH_CUDA(o, cudaStreamWaitEvent(o.stream, o.evD2H, 0));
        }
    }
    o.processedFFT = o.processedIFFT = o.processedTilt = 1;
    o.processedOverlap = o.modeCount > 0;
    o.metricsValid = 0;
    r = applyBasis(o);
    if (r) return r;
    (void)g;
    // the frame source of this batch, for the Fourier planes on request
    o.lastFwd = fp;
    if (!o.framesOnDevice) {
        o.lastFwd.frames = o.dFrames.ptr;
        o.lastFwd.frameWidth = g.W;
        o.lastFwd.frameStride = (long long)P * g.H * g.W;
        for (int p = 0; p < P; p++) { o.lastFwd.cx[p] = 0; o.lastFwd.cy[p] = p * g.H; }
    } else {
        o.lastFwd.frames = o.frames;
        o.lastFwd.frameWidth = o.cfg.frameWidth;
        o.lastFwd.frameStride = (long long)o.cfg.frameWidth * o.cfg.frameHeight;
        for (int p = 0; p < P; p++) { o.lastFwd.cx[p] = g.cx[p]; o.lastFwd.cy[p] = g.cy[p]; }
    }
    o.lastFwd.frameCount = B * o.avgCount;
    o.lastFwd.frameOffset = 0;
    {
        // the excluded disk of the Fourier-plane analysis: radius 2 k0 sin(aperture)
        // in float32 (digHolo.cpp:6936-6939)
        const Config& cc = o.useSnaps ? o.fftSnap : o.cfg;
        const float k0 = 2 * PI_F / cc.wavelengthCentre;
        const float R = 2 * k0 * sinf(cc.apertureSize * UNIT_ANGLE);
        o.lastFourierR2 = R * R;
    }
    o.lastFwdValid = 1;
    o.fourierValid = 0;
    if (planNeeded) {
        DhFwdParams pfp = o.lastFwd;
        pfp.frameCount = B;
        r = planBatch(o, pfp, ip);
        if (r) return r;
        r = applyBasis(o);
        if (r) return r;
    }
    if (earlyCoefs) {
        // the coefficients are already on their way (the stream waits for them)
        DH_CUDA(o, cudaStreamSynchronize(o.stream));
        return objCheckStatus(o);
    }
    if (syncCoefs) return objCoefsToHost(o);
    return ERR_SUCCESS;
}

// The batch path with caller-owned outputs and an external window scratch
// (digHoloB200ProcessBatchNoAlloc).  Allocates nothing: the handle's tables
// must already match the configuration.
int objProcessNoAlloc(Object& o, const void* frames, int B, int u16, float2* window, size_t windowBytes,
                      float2* coefs, short* fieldR, short* fieldI, float* stats) {
    std::lock_guard<std::mutex> guard(o.lock);
    if (o.device < 0 || !o.preparedValid || !window)
        return fail(o, ERR_ERROR, "no-alloc path: process one batch with this configuration first (that call allocates)");
    cudaSetDevice(o.device);
    Config a = o.cfg, b = o.preparedCfg;
    a.batchCount = b.batchCount = 0;
    if (a.fftWindowSizeX <= 0) a.fftWindowSizeX = a.frameWidth / a.polCount;
    if (a.fftWindowSizeY <= 0) a.fftWindowSizeY = a.frameHeight;
    if (memcmp(&a, &b, sizeof(Config)) != 0)
        return fail(o, ERR_ERROR, "no-alloc path: configuration changed since the handle was prepared");
    if (o.avgCount > 1)
        return fail(o, ERR_INVALIDARGUMENT, "no-alloc path: frame averaging (avgCount > 1) needs digHoloProcessBatch");
    if (o.cfg.basisType == 1 || (o.cfg.basisType == 2 && !o.basisCustom.empty()))
        return fail(o, ERR_INVALIDARGUMENT, "no-alloc path: returns Hermite-Gaussian coefficients only (basis type 0)");
    const Geometry& g = o.geo;
    const int P = o.polCount;
    if ((size_t)B * P * g.w * g.h * sizeof(float2) > windowBytes)
        return fail(o, ERR_INVALIDDIMENSION, "no-alloc path: frameCount * polCount * w * h * 8 bytes exceeds the 8 MiB window scratch");
    if (o.cfg.maxMG > 0) {
        if (!coefs) return fail(o, ERR_NULLPOINTER, "no-alloc path: coefficient buffer is null");
        if (o.basisMG != o.cfg.maxMG || o.basisNx != g.nx || o.basisNy != g.ny || o.basisPolCount != P)
            return fail(o, ERR_ERROR, "no-alloc path: basis not prepared for this configuration");
    }
    if (!isDevicePointer(frames) || (reinterpret_cast<uintptr_t>(frames) % 16))
        return fail(o, ERR_INVALIDARGUMENT, "no-alloc path: frames must be a 16-byte aligned device pointer");
    const int saveU16 = o.framesU16;
    o.framesU16 = u16;
    DhFwdParams fp;
    forwardParams(o, fp);
    o.framesU16 = saveU16;
    fp.frames = frames;
    fp.frameWidth = o.cfg.frameWidth;
    fp.frameStride = (long long)o.cfg.frameWidth * o.cfg.frameHeight;
    for (int p = 0; p < P; p++) { fp.cx[p] = g.cx[p]; fp.cy[p] = g.cy[p]; }
    fp.frameCount = B;
    fp.frameOffset = 0;
    fp.window = window;
    DhInvParams ip;
    inverseParams(o, ip, o.cfg.maxMG > 0);
    {
        const int rc = calParams(o, ip, true);
        if (rc) return rc;
    }
    ip.window = window;
    ip.frameCount = B;
    ip.fieldR = fieldR;
    ip.fieldI = fieldI;
    ip.field32 = nullptr;
    ip.stats = stats;
    ip.statsStride = B + 1;
    ip.coefs = o.cfg.maxMG > 0 ? coefs : nullptr;
    if (!ip.coefs) ip.maxMG = 0;
    cudaError_t fe = launchForward(o, fp, false);
    if (fe == cudaErrorMemoryAllocation)
        return fail(o, ERR_MEMORYALLOCATION, "no-alloc path: the Fourier-plane buffer was sized for a smaller batch");
    if (fe != cudaSuccess) return failCuda(o, fe, "no-alloc forward kernel launch");
    // the full-plane forward wrote this call's planes over the last batch's:
    // a later Fourier-plane request recomputes them from that batch's frames
    if (o.lastForwardKernel == 5) o.fourierValid = 0;
    fe = launchInverse(o, ip, false);
    if (fe == cudaErrorMemoryAllocation)
        return fail(o, ERR_MEMORYALLOCATION, "no-alloc path: the band scratch was sized for a smaller batch");
    DH_CUDA(o, fe);
    return ERR_SUCCESS;
}

// Inverse stage on another window buffer of the current geometry: the float
// field -conj(A R) to field32, the int16 field and statistics to scratch, no
// overlap.  The beam-centre derivative fields of the adjoint use it.
int objInverseAux(Object& o, const float2* window, int frameCount, float2* field32, short* scratchR, short* scratchI,
                  float* scratchStats) {
    DhInvParams ip;
    inverseParams(o, ip, 0);
    {
        const int rc = calParams(o, ip);
        if (rc) return rc;
    }
    ip.frameCount = frameCount;
    ip.statsStride = frameCount + 1;
    ip.window = window;
    ip.field32 = field32;
    ip.fieldR = scratchR;
    ip.fieldI = scratchI;
    ip.stats = scratchStats;
    ip.fieldsOnly = 1;
    const int k = o.lastInverseKernel, ov = o.lastOverlapKernel;
    DH_CUDA(o, launchInverse(o, ip));
    o.lastInverseKernel = k;
    o.lastOverlapKernel = ov;
    return ERR_SUCCESS;
}

// Unquantised float HG modes [pol][modes][n] on the reconstructed-plane axes
// for the current waists (the FP64 recurrence of digHolo.cpp:1269-1484).
int objBasisFloat(Object& o, int modes, float* outX, float* outY, short* scratch16, float* scratchScale) {
    const Config& c = o.cfg;
    const Geometry& g = o.geo;
    const int P = o.polCount;
    DhBasisParams jobs[4];
    int n = 0;
    for (int p = 0; p < P; p++) {
        float w = c.waist[c.polLockBasisWaist ? 0 : p];
        if (w == 0) w = 400e-6f;
        jobs[n++] = DhBasisParams{o.dX.as<float>(), g.nx, modes, (double)w, scratch16, scratchScale,
                                  outX + (size_t)p * modes * g.nx, 0};
        jobs[n++] = DhBasisParams{o.dY.as<float>(), g.ny, modes, (double)w, scratch16, scratchScale,
                                  outY + (size_t)p * modes * g.ny, 0};
    }
    DH_CUDA(o, dh_launch_basis_jobs(jobs, n, o.stream));
    return ERR_SUCCESS;
}

// The batch path for one AutoAlign evaluation: outputs stay on the device.
int objProcessForAlign(Object& o) {
    int r = objProcessBatch(o, 0);
    if (r) return r;
    return ERR_SUCCESS;
}

int objCoefsToHost(Object& o) {
    if (o.modeCount <= 0 || !o.dCoefs.ptr) {
        DH_CUDA(o, cudaStreamSynchronize(o.stream));
        return objCheckStatus(o);
    }
    const size_t n = (size_t)o.batchCount * o.polCount * objOutputModes(o) * sizeof(float2);
    if (!o.hCoefs.ensure(n)) return fail(o, ERR_MEMORYALLOCATION, "host coefficient buffer");
    DH_CUDA(o, cudaMemcpyAsync(o.hCoefs.ptr, objOutputCoefs(o), n, cudaMemcpyDeviceToHost, o.stream));
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    return objCheckStatus(o);
}

// Individual steps (digHoloProcessFFT/IFFT/RemoveTilt/BasisExtractCoefs).
// The forward kernel fuses the FFT with the window copy of the IFFT step, and
// the inverse kernel fuses the IFFT with the tilt removal and the overlap, so
// each step runs the fused kernels up to and including its own work.
int objFFT(Object& o) {
    std::lock_guard<std::mutex> guard(o.lock);
    int r = prepare(o);
    if (r) return r;
    o.processedFFT = 1;
    o.processedIFFT = o.processedTilt = o.processedOverlap = 0;
    return ERR_SUCCESS;
}

static int runStages(Object& o, int withInverse, int withOverlap) {
    int r = prepare(o);
    if (r) return r;
    if (withOverlap) {
        r = updateBasis(o);
        if (r) return r;
        if (o.modeCount > 0)
            DH_CUDA(o, o.dCoefs.ensure((size_t)o.batchCount * o.polCount * o.modeCount * sizeof(float2)));
    }
    DhFwdParams fp;
    forwardParams(o, fp);
    r = stageFrames(o, 0, o.batchCount * o.avgCount, fp, 0);
    if (r) return r;
    DhInvParams ip;
    inverseParams(o, ip, withOverlap);
    r = calParams(o, ip);
    if (r) return r;
    if (!withInverse) ip.fieldR = nullptr;
    r = o.avgCount > 1 ? launchAveraged(o, fp, ip) : launchChunk(o, fp, ip, 0, o.batchCount);
    if (r) return r;
    if (withOverlap) {
        r = applyBasis(o);
        if (r) return r;
    }
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    return ERR_SUCCESS;
}

int objIFFT(Object& o) {
    std::lock_guard<std::mutex> guard(o.lock);
    int r = runStages(o, 0, 0);
    if (r) return r;
    o.processedFFT = o.processedIFFT = 1;
    o.processedTilt = o.processedOverlap = 0;
    return ERR_SUCCESS;
}

int objApplyTilt(Object& o) {
    std::lock_guard<std::mutex> guard(o.lock);
    int r = runStages(o, 1, 0);
    if (r) return r;
    o.processedFFT = o.processedIFFT = o.processedTilt = 1;
    o.processedOverlap = 0;
    return ERR_SUCCESS;
}

int objOverlap(Object& o) {
    std::lock_guard<std::mutex> guard(o.lock);
    if (o.cfg.maxMG <= 0) {
        o.modeCount = 0;
        return ERR_SUCCESS;
    }
    int r = runStages(o, 1, 1);
    if (r) return r;
    o.processedFFT = o.processedIFFT = o.processedTilt = o.processedOverlap = 1;
    return objCoefsToHost(o);
}

// Fourier planes of the last batch, their statistics and batch-sum intensity
// (computed once per batch from the frames it was processed from; those
// frames must still be valid, as for digHoloProcessBatch), copied to the
// host mirrors; the plane only when withPlane.
int objFourierToHost(Object& o, int withPlane) {
    if (!o.lastFwdValid) return fail(o, ERR_NULLPOINTER, "no batch has been processed");
    const Geometry& g = o.geo;
    const int B = o.lastFwd.frameCount, P = o.polCount;
    const size_t Nx = (size_t)g.W / 2 + 1;
    const size_t planeN = (size_t)B * P * g.H * Nx;
    const size_t statsN = (size_t)ANALYSIS_COUNT * P * (B + 1);
    const size_t sumN = (size_t)P * g.W * g.H;
    if (!o.fourierValid) {
        DH_CUDA(o, o.dFourier.ensure(planeN * sizeof(float2)));
        DH_CUDA(o, o.dFftStats.ensure(statsN * sizeof(float)));
        DH_CUDA(o, o.dFftBatchSum.ensure(sumN * sizeof(float)));
        DH_CUDA(o, cudaMemsetAsync(o.dFftBatchSum.ptr, 0, sumN * sizeof(float), o.stream));
        DhFourierParams q;
        memset(&q, 0, sizeof(q));
        q.f = o.lastFwd;
        q.plane = o.dFourier.as<float2>();
        q.kx = o.dKx.as<float>();
        q.ky = o.dKy.as<float>();
        q.r2 = o.lastFourierR2;
        q.stats = o.dFftStats.as<float>();
        q.batchSum = o.dFftBatchSum.as<float>();
        DH_CUDA(o, dh_launch_fourier_full(q, o.stream));
        o.fourierValid = 1;
    }
    if (!o.hFftStats.ensure(statsN * sizeof(float))) return fail(o, ERR_MEMORYALLOCATION, "host Fourier stats buffer");
    if (!o.hFftBatchSum.ensure(sumN * sizeof(float))) return fail(o, ERR_MEMORYALLOCATION, "host Fourier batch-sum buffer");
    DH_CUDA(o, cudaMemcpyAsync(o.hFftStats.ptr, o.dFftStats.ptr, statsN * sizeof(float), cudaMemcpyDeviceToHost, o.stream));
    DH_CUDA(o, cudaMemcpyAsync(o.hFftBatchSum.ptr, o.dFftBatchSum.ptr, sumN * sizeof(float), cudaMemcpyDeviceToHost, o.stream));
    if (withPlane) {
        if (!o.hFourier.ensure(planeN * sizeof(float2))) return fail(o, ERR_MEMORYALLOCATION, "host Fourier plane buffer");
        DH_CUDA(o, cudaMemcpyAsync(o.hFourier.ptr, o.dFourier.ptr, planeN * sizeof(float2), cudaMemcpyDeviceToHost, o.stream));
    }
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    o.hKx = g.kx;
    o.hKy = g.ky;
    return objCheckStatus(o);
}

int objStatsToHost(Object& o) {
    const int B = o.batchCount, P = o.polCount;
    const Geometry& g = o.geo;
    const size_t npix = (size_t)g.nx * g.ny;
    const size_t n = (size_t)ANALYSIS_COUNT * P * (B + 1);
    // host layout [parameter][pol][batch x avg + 1] (digHolo.cpp:7619): with
    // frame averaging the batch entries and the aggregate fill the first B + 1
    const int SA = B * std::max(1, o.avgCount) + 1;
    if (!o.hStats.ensure((size_t)ANALYSIS_COUNT * P * SA * sizeof(float)))
        return fail(o, ERR_MEMORYALLOCATION, "host stats buffer");
    // per polarisation W H floats, the plane in the first nx ny (the reference
    // sizes every batch-sum plane by the FFT window, digHolo.cpp:7655)
    const size_t stride = std::max((size_t)g.W * g.H, npix);
    if (!o.hBatchSum.ensure((size_t)P * stride * sizeof(float))) return fail(o, ERR_MEMORYALLOCATION, "host batch-sum buffer");
    DH_CUDA(o, o.dFieldsC64.ensure((size_t)P * npix * sizeof(float)));
    DH_CUDA(o, dh_launch_batchsum(o.dFieldR.as<short>(), o.dFieldI.as<short>(), o.dStats.as<float>(), B + 1, P, B,
                                  (int)npix, o.dFieldsC64.as<float>(), o.stream));
    DH_CUDA(o, cudaMemcpyAsync(o.hStats.ptr, o.dStats.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, o.stream));
    DH_CUDA(o, cudaMemcpyAsync(o.hBatchSum.ptr, o.dFieldsC64.ptr, (size_t)P * npix * sizeof(float), cudaMemcpyDeviceToHost, o.stream));
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    // Aggregate column [B]: the analysis of the summed intensity (digHolo.cpp:2519-2568).
    float* s = o.hStats.as<float>();
    const float* sum = o.hBatchSum.as<float>();
    const int S = B + 1;
    const float yShift = fabsf((g.y[1] - g.y[0]) * (float)g.ny);
    const float dA = fabsf(g.x[2] - g.x[1]) * fabsf(g.y[2] - g.y[1]);
    for (int p = 0; p < P; p++) {
        double Pw = 0, cx = 0, cy = 0, cyw = 0, e4 = 0, mx = 0;
        int mxIdx = -1;
        for (int y = 0; y < g.ny; y++)
            for (int x = 0; x < g.nx; x++) {
                const double I = sum[(size_t)p * npix + (size_t)y * g.nx + x];
                Pw += I;
                cx += g.x[x] * I;
                cy += g.y[y] * I;
                cyw += (g.y[y] + (g.y[y] < 0 ? yShift : 0.f)) * I;
                e4 += I * I;
                // the reference compares the summed intensity against an index
                // vector already advanced to the next block of 8 (digHolo.cpp:2533-2561)
                const int idx = 2 * y * g.nx + x + 8;
                if (I >= mx) { mx = I; mxIdx = idx; }
            }
        const int per = P * S;
        const int col = p * S + B;
        s[0 * per + col] = (float)Pw;
        s[1 * per + col] = (float)(cx / Pw);
        s[2 * per + col] = (float)(cy / Pw);
        s[3 * per + col] = (float)(32767.0 / sqrt(mx));
        memcpy(&s[4 * per + col], &mxIdx, sizeof(int));
        s[5 * per + col] = (float)(dA * (Pw * Pw / e4));
        s[6 * per + col] = (float)(cyw / Pw);
    }
    if (SA != S) {   // spread the rows to the averaged stride (last first: the moves go up)
        for (int r = ANALYSIS_COUNT * P - 1; r >= 0; r--) {
            memmove(s + (size_t)r * SA, s + (size_t)r * S, S * sizeof(float));
            memset(s + (size_t)r * SA + S, 0, (SA - S) * sizeof(float));
        }
    }
    // spread the polarisations to their strides (last first: the moves go up)
    float* sb = o.hBatchSum.as<float>();
    for (int p = P - 1; p >= 0; p--) {
        if (p > 0) memmove(sb + (size_t)p * stride, sb + (size_t)p * npix, npix * sizeof(float));
        memset(sb + (size_t)p * stride + npix, 0, (stride - npix) * sizeof(float));
    }
    return ERR_SUCCESS;
}

int objFieldsToHost(Object& o, int complexOut) {
    const Geometry& g = o.geo;
    const size_t npix = (size_t)g.nx * g.ny;
    const size_t n = (size_t)o.batchCount * o.polCount * npix;
    if (complexOut) {
        if (!o.hFields.ensure(n * sizeof(float2))) return fail(o, ERR_MEMORYALLOCATION, "host field buffer");
        DH_CUDA(o, o.dFieldsC64.ensure(n * sizeof(float2)));
        DH_CUDA(o, dh_launch_fields_to_c64(o.dFieldR.as<short>(), o.dFieldI.as<short>(), o.dStats.as<float>(),
                                           o.batchCount + 1, o.polCount, o.batchCount, (int)npix,
                                           o.dFieldsC64.as<float2>(), o.stream));
        DH_CUDA(o, cudaMemcpyAsync(o.hFields.ptr, o.dFieldsC64.ptr, n * sizeof(float2), cudaMemcpyDeviceToHost, o.stream));
    } else {
        if (!o.hFieldR.ensure(2 * n * sizeof(short))) return fail(o, ERR_MEMORYALLOCATION, "host int16 field buffer");
        DH_CUDA(o, cudaMemcpyAsync(o.hFieldR.ptr, o.dFieldR.ptr, n * sizeof(short), cudaMemcpyDeviceToHost, o.stream));
        DH_CUDA(o, cudaMemcpyAsync(o.hFieldR.as<short>() + n, o.dFieldI.ptr, n * sizeof(short), cudaMemcpyDeviceToHost, o.stream));
    }
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    return objStatsToHost(o);
}

int objWindowToHost(Object& o) {
    const Geometry& g = o.geo;
    const size_t n = (size_t)o.batchCount * o.polCount * g.w * g.h;
    if (!o.hWindow.ensure(n * sizeof(float2))) return fail(o, ERR_MEMORYALLOCATION, "host window buffer");
    DH_CUDA(o, cudaMemcpyAsync(o.hWindow.ptr, o.dWindow.ptr, n * sizeof(float2), cudaMemcpyDeviceToHost, o.stream));
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    return ERR_SUCCESS;
}

}  // namespace dh
