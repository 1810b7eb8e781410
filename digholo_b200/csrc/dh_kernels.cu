// sm_100a kernels for the digHolo batch path.
//
//   k_forward : frame window -> pruned R2C FFT -> Fourier window ops
//               (replaces convert_int16tofloat32 digHolo.cpp:1201, the FFTW
//               r2c batch digHolo.cpp:7184-7260 and digHoloCopyWindow
//               digHolo.cpp:1808-2122)
//   k_inverse : window IFFT -> field statistics -> reference wave, -conj,
//               int16 rounding -> separable HG overlap
//               (replaces the FFTW c2c backward digHolo.cpp:8734,
//               digHoloFieldAnalysis digHolo.cpp:2354, applyTilt16
//               digHolo.cpp:2701 and overlapFieldSeparable16 digHolo.cpp:2149)
//   k_basis   : FP64 Hermite-Gaussian recurrence -> int16 modes + scales
//               (replaces HGbasisXY1D digHolo.cpp:1269-1484)
//   k_fields_to_c64 : int16 field -> complex64 x 1/scale (digHoloGetFields,
//               digHolo.cpp:4930-4981)
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"

using namespace dh;

namespace {

constexpr int FWD_THREADS = 256;
constexpr int INV_THREADS = 512;
// Row-FFT staging budget of the forward kernel (complex elements).
constexpr int FWD_ROWBUF_ELEMS = 4096;

__device__ __forceinline__ int wrapMod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ void load8(const void* frames, int u16, long long idx, float* v) {
    if (u16) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(frames) + idx));
        v[0] = (float)(q.x & 0xFFFFu); v[1] = (float)(q.x >> 16);
        v[2] = (float)(q.y & 0xFFFFu); v[3] = (float)(q.y >> 16);
        v[4] = (float)(q.z & 0xFFFFu); v[5] = (float)(q.z >> 16);
        v[6] = (float)(q.w & 0xFFFFu); v[7] = (float)(q.w >> 16);
    } else {
        const float4* s = reinterpret_cast<const float4*>(static_cast<const float*>(frames) + idx);
        const float4 a = __ldg(s), b = __ldg(s + 1);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    }
}

}  // namespace

// One block per (frame, polarisation, column chunk).  The window rows are
// staged in blocks of RB rows, transformed as packed half-length complex
// FFTs, and only the kx columns of the IFFT window are kept (R2C split
// post-processing).  The kept columns are then transformed along y and only
// the ky rows of the IFFT window are kept.
__global__ void __launch_bounds__(FWD_THREADS) k_forward(DhFwdParams p) {
    extern __shared__ float2 sm[];
    const int W = 1 << p.logW, H = 1 << p.logH;
    const int logN = p.logW - 1, N = W >> 1;
    const int WC = p.colChunk;
    const int chunks = p.w / WC;
    int unit = blockIdx.x;
    const int chunk = unit % chunks;
    unit /= chunks;
    const int pol = unit % p.polCount;
    const int frame = unit / p.polCount;
    int RB = FWD_ROWBUF_ELEMS / N;
    if (RB > H) RB = H;
    float2* rowbuf = sm;
    float2* colbuf = sm + RB * N;
    const int kStart = p.sx0[pol] + chunk * WC;
    const long long base = (long long)frame * p.frameStride + (long long)p.cy[pol] * p.frameWidth + p.cx[pol];
    const int vecPerRow = W >> 3;

    for (int r0 = 0; r0 < H; r0 += RB) {
        for (int e = threadIdx.x; e < RB * vecPerRow; e += blockDim.x) {
            const int r = e / vecPerRow, v = e - r * vecPerRow;
            float x[8];
            load8(p.frames, p.inputU16, base + (long long)(r0 + r) * p.frameWidth + v * 8, x);
            float2* dst = rowbuf + r * N;
#pragma unroll
            for (int q = 0; q < 4; q++) dst[bitrev(v * 4 + q, logN)] = make_float2(x[2 * q], x[2 * q + 1]);
        }
        __syncthreads();
        fft_dit(rowbuf, RB, N, 1, logN, false, false, p.twiddle);
        for (int e = threadIdx.x; e < RB * WC; e += blockDim.x) {
            const int r = e / WC, c = e - r * WC;
            const int k = kStart + c;
            const float2 zk = rowbuf[r * N + (k & (N - 1))];
            const float2 zc = cconj(rowbuf[r * N + ((N - k) & (N - 1))]);
            const float2 even = cscale(cadd(zk, zc), 0.5f);
            const float2 d = csub(zk, zc);
            const float2 odd = make_float2(0.5f * d.y, -0.5f * d.x);  // -i/2 (zk - zc)
            const float2 wk = __ldg(&p.twiddle[k << (TW_LOG - p.logW)]);
            colbuf[bitrev(r0 + r, p.logH) * WC + c] = cadd(even, cmul(wk, odd));
        }
        __syncthreads();
    }
    fft_dit(colbuf, WC, 1, WC, p.logH, false, true, p.twiddle);

    float2 bc = make_float2(1.0f, 0.0f);
    if (p.batchCal && p.batchCalCount > 0)
        bc = p.batchCal[pol * p.batchCalCount + ((p.frameOffset + frame) % p.batchCalCount)];
    const float kx0 = p.kx0[pol], ky0 = p.ky0[pol], r02 = p.r02[pol];
    const float bcx = p.bcx[pol], bcy = p.bcy[pol];
    for (int e = threadIdx.x; e < p.h * WC; e += blockDim.x) {
        const int j = e / WC, c = e - j * WC;
        const int jSY = j + p.sy[pol];
        const int row = wrapMod(jSY + H / 2, H);
        float2 Y = colbuf[row * WC + c];
        Y = cmul(Y, bc);
        const float kx = p.kxAxis[kStart + c];
        const float ky = p.kyAxis[row];
        const float shift = jSY < 0 ? p.kyShift : (jSY > H ? -p.kyShift : 0.0f);
        // the mask test in float32 as digHolo.cpp:1984-2019 evaluates it
        const float dky = __fsub_rn(ky, __fadd_rn(ky0, shift));
        const float dkx = __fsub_rn(kx, kx0);
        const float dr2 = __fadd_rn(__fmul_rn(dkx, dkx), __fmul_rn(dky, dky));
        float env = 1.0f;
        if (p.fillFactor) env = xcsc(kx * p.halfPixel) * xcsc(ky * p.halfPixel);
        const float normF = (dr2 <= r02) ? env * p.norm : 0.0f;
        const float arg = __fadd_rn(__fmul_rn(bcx, kx), __fmul_rn(ky, bcy));
        float sn, cs;
        sincosf(arg, &sn, &cs);
        const float2 adj = make_float2(cs * normF, sn * normF);
        const size_t o = ((size_t)(frame * p.polCount + pol) * p.h + j) * p.w + chunk * WC + c;
        p.window[o] = cmul(Y, adj);
    }
}

namespace {

struct Stat6 {
    float maxI;
    int maxIdx;
    float P, cx, cy, cyw, e4;
};

__device__ __forceinline__ void statCombine(Stat6& a, const Stat6& b) {
    if (b.maxI > a.maxI || (b.maxI == a.maxI && b.maxIdx > a.maxIdx)) { a.maxI = b.maxI; a.maxIdx = b.maxIdx; }
    a.P += b.P; a.cx += b.cx; a.cy += b.cy; a.cyw += b.cyw; a.e4 += b.e4;
}

__device__ Stat6 blockReduceStat(Stat6 s, Stat6* scratch) {
    for (int off = 16; off > 0; off >>= 1) {
        Stat6 o;
        o.maxI = __shfl_down_sync(0xffffffffu, s.maxI, off);
        o.maxIdx = __shfl_down_sync(0xffffffffu, s.maxIdx, off);
        o.P = __shfl_down_sync(0xffffffffu, s.P, off);
        o.cx = __shfl_down_sync(0xffffffffu, s.cx, off);
        o.cy = __shfl_down_sync(0xffffffffu, s.cy, off);
        o.cyw = __shfl_down_sync(0xffffffffu, s.cyw, off);
        o.e4 = __shfl_down_sync(0xffffffffu, s.e4, off);
        statCombine(s, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) scratch[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        Stat6 t = scratch[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); i++) statCombine(t, scratch[i]);
        scratch[0] = t;
    }
    __syncthreads();
    return scratch[0];
}

}  // namespace

// One block per (frame, polarisation).
// field x calibration with the reference's complex product, real part fused
// (cmul, digHolo.cpp:885-892)
__device__ __forceinline__ float2 calMul(float2 a, float2 c) {
    return make_float2(__fmaf_rn(a.x, c.x, -__fmul_rn(a.y, c.y)), __fmaf_rn(a.x, c.y, __fmul_rn(a.y, c.x)));
}

__global__ void __launch_bounds__(INV_THREADS) k_inverse(DhInvParams p) {
    extern __shared__ float2 sm[];
    const int unit = blockIdx.x;
    const int pol = unit % p.polCount;
    const int frame = unit / p.polCount;
    const int w = 1 << p.logw, h = 1 << p.logh;
    const int W = 1 << p.logW, H = 1 << p.logH;
    const int lognx = p.lowres ? p.logw : p.logW;
    const int logny = p.lowres ? p.logh : p.logH;
    const int nx = 1 << lognx, ny = 1 << logny;
    const int npix = nx * ny;
    const int ld = nx + 1;                           // padded row stride of the field in shared memory
    float2* fld = sm;
    float2* colbuf = fld + (size_t)ny * ld;          // full-res only: H * w
    float* extra = reinterpret_cast<float*>(colbuf + (p.lowres ? 0 : H * w));
    const float2* win = p.window + (size_t)unit * h * w;

    if (p.lowres) {
        for (int e = threadIdx.x; e < h * w; e += blockDim.x) {
            const int j = e >> p.logw, c = e & (w - 1);
            fld[bitrev(j, p.logh) * ld + bitrev(c, p.logw)] = win[e];
        }
        __syncthreads();
        fft_dit(fld, h, ld, 1, p.logw, true, false, p.twiddle);
        fft_dit(fld, w, 1, ld, p.logh, true, true, p.twiddle);
    } else {
        for (int e = threadIdx.x; e < H * w; e += blockDim.x) colbuf[e] = make_float2(0.f, 0.f);
        for (int e = threadIdx.x; e < ny * ld; e += blockDim.x) fld[e] = make_float2(0.f, 0.f);
        __syncthreads();
        const int syp = p.sy[pol];
        for (int e = threadIdx.x; e < h * w; e += blockDim.x) {
            const int j = e >> p.logw, c = e & (w - 1);
            const int row = wrapMod(j + syp + H / 2, H);
            colbuf[bitrev(row, p.logH) * w + c] = win[e];
        }
        __syncthreads();
        fft_dit(colbuf, w, 1, w, p.logH, true, true, p.twiddle);
        const int sx0 = p.sx0[pol];
        for (int e = threadIdx.x; e < H * w; e += blockDim.x) {
            const int y = e >> p.logw, c = e & (w - 1);
            fld[y * ld + bitrev((sx0 + c) & (W - 1), p.logW)] = colbuf[e];
        }
        __syncthreads();
        fft_dit(fld, H, ld, 1, p.logW, true, false, p.twiddle);
    }
    if (p.refCal) {
        // reference-wave calibration of the IFFT output (digHolo.cpp:8736-8758, 8770-8782)
        const float2* cal = p.refCal + (size_t)pol * npix;
        for (int e = threadIdx.x; e < npix; e += blockDim.x) {
            const int y = e >> lognx, x = e & (nx - 1);
            fld[y * ld + x] = calMul(fld[y * ld + x], cal[e]);
        }
        __syncthreads();
    }

    // Field statistics over the whole untilted field (windowRadius = 0,
    // digHolo.cpp:8866-8870): power, centre of mass, max|E|, E^4.
    Stat6* scratch = reinterpret_cast<Stat6*>(extra);
    const float inv = (float)(1.0 / ((double)nx * (double)ny));
    const float yShift = fabsf((p.yAxis[1] - p.yAxis[0]) * (float)ny);
    Stat6 st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int y = e >> lognx, x = e & (nx - 1);
        const float2 a = fld[y * ld + x];
        const float I0 = fmaf(a.x, a.x, a.y * a.y);
        const float I = I0 * inv;
        const int idx = 2 * y * nx + x;
        if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
        const float yv = p.yAxis[y];
        st.P += I;
        st.cx = fmaf(p.xAxis[x], I, st.cx);
        st.cy = fmaf(yv, I, st.cy);
        st.cyw = fmaf(yv + (yv < 0.f ? yShift : 0.f), I, st.cyw);
        st.e4 = fmaf(I, I, st.e4);
    }
    st = blockReduceStat(st, scratch);
    const float maxAbs = sqrtf(st.maxI);
    const float scale = (float)(32767.0 / (double)maxAbs);
    if (threadIdx.x == 0) {
        const int S = p.statsStride;
        float* s = p.stats;
        const int col = pol * S + frame;
        const int per = p.polCount * S;
        s[0 * per + col] = st.P;
        s[1 * per + col] = st.cx / st.P;
        s[2 * per + col] = st.cy / st.P;
        s[3 * per + col] = scale;
        s[4 * per + col] = __int_as_float(st.maxIdx);
        s[5 * per + col] = p.dA * (st.P * st.P / st.e4);
        s[6 * per + col] = st.cyw / st.P;
    }

    // Reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833).
    const short* ref = p.refWave + (size_t)pol * 2 * (nx + ny);
    const float K = (float)(1.0 / (16383.0 * 16383.0));
    const size_t fieldOff = (size_t)unit * npix;
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int y = e >> lognx, x = e & (nx - 1);
        const int xr = ref[x], xi = ref[nx + x];
        const int yr = ref[2 * nx + y], yi = ref[2 * nx + ny + y];
        const float adjR = (float)(yr * xr - yi * xi) * K;
        const float adjI = (float)(yr * xi + yi * xr) * K;
        const float2 a = fld[y * ld + x];
        const float vr = __fsub_rn(__fmul_rn(a.y, adjI), __fmul_rn(a.x, adjR));
        const float vi = __fadd_rn(__fmul_rn(a.x, adjI), __fmul_rn(a.y, adjR));
        if (p.field32) {
            // float path: the same -conj(A . ref) with the unquantised wave
            const float* rf = p.refWaveF + (size_t)pol * 2 * (nx + ny);
            const float2 rx = make_float2(rf[x], rf[nx + x]);
            const float2 ry = make_float2(rf[2 * nx + y], rf[2 * nx + ny + y]);
            const float2 v = cmul(a, cmul(ry, rx));
            p.field32[fieldOff + e] = make_float2(-v.x, v.y);
        }
        const float fr = rintf(scale * vr), fi = rintf(scale * vi);
        // float -> int32 with the x86 convention (NaN / overflow -> INT_MIN),
        // then saturate to int16 (digHolo.cpp:2822-2829)
        const int ir = (fr >= -2147483648.0f && fr < 2147483648.0f) ? (int)fr : INT32_MIN;
        const int ii = (fi >= -2147483648.0f && fi < 2147483648.0f) ? (int)fi : INT32_MIN;
        const short sr = (short)max(-32768, min(32767, ir));
        const short si = (short)max(-32768, min(32767, ii));
        p.fieldR[fieldOff + e] = sr;
        p.fieldI[fieldOff + e] = si;
        fld[y * ld + x] = make_float2((float)sr, (float)si);
    }
    __syncthreads();

    if (p.maxMG <= 0) return;

    // Separable overlap on the int16 field (digHolo.cpp:2149-2341):
    // T[y][m] = sum_x F[y][x] Hx[m][x];  c_mn = sum_y Hy[n][y] T[y][m].
    const int G = p.maxMG;
    float* hx = extra;                 // [G][nx]
    float* hy = hx + G * nx;           // [G][ny]
    float2* T = reinterpret_cast<float2*>(hy + G * ny);   // [ny][G]
    const short* gx = p.hgX + (size_t)pol * G * nx;
    const short* gy = p.hgY + (size_t)pol * G * ny;
    for (int e = threadIdx.x; e < G * nx; e += blockDim.x) hx[e] = (float)gx[e];
    for (int e = threadIdx.x; e < G * ny; e += blockDim.x) hy[e] = (float)gy[e];
    __syncthreads();
    for (int e = threadIdx.x; e < ny * G; e += blockDim.x) {
        const int m = e >> logny, y = e & (ny - 1);
        const float2* row = fld + y * ld;
        const float* hm = hx + m * nx;
        float ar = 0.f, ai = 0.f;
        for (int x = 0; x < nx; x++) {
            const float2 f = row[x];
            const float hv = hm[x];
            ar = fmaf(f.x, hv, ar);
            ai = fmaf(f.y, hv, ai);
        }
        T[y * G + m] = make_float2(ar, ai);
    }
    __syncthreads();
    const float fieldScale = 1.0f / scale;
    const float* sxp = p.hgScaleX + pol * G;
    const float* syp = p.hgScaleY + pol * G;
    for (int mode = threadIdx.x; mode < p.modeCount; mode += blockDim.x) {
        // mode -> (m, n): group g, n = mode - g(g+1)/2, m = g - n (digHolo.cpp:1245-1265)
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2;
        const int m = g - n;
        const float* hn = hy + n * ny;
        float cr = 0.f, ci = 0.f;
        for (int y = 0; y < ny; y++) {
            const float2 t = T[y * G + m];
            cr = fmaf(hn[y], t.x, cr);
            ci = fmaf(hn[y], t.y, ci);
        }
        const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
        p.coefs[(size_t)frame * p.polCount * p.modeCount + pol * p.modeCount + mode] = make_float2(cr * ms, ci * ms);
    }
}

// Low-resolution fields of any size that is a multiple of 16 (48, 80, 96,
// 112 ...: the sides FFTW transforms directly in the reference, digHolo.cpp:8734),
// one block per (frame, polarisation): the h x w inverse DFT as two direct
// passes through shared memory (rows against exp(+2 pi i kx x / w), then
// columns against exp(+2 pi i ky y / h), twiddles from sincospi in double
// rounded once), then the statistics, the reference wave, int16 rounding and
// the separable overlap of k_inverse.
constexpr int DFT_THREADS = 256;

struct DftSmem {
    size_t win, tmp, tw, scratch, total;
};
__host__ __device__ inline DftSmem dftSmem(int w, int h, int G) {
    DftSmem s;
    const size_t plane = sizeof(float2) * (size_t)h * (w + 1);
    size_t ov = G > 0 ? sizeof(float) * (size_t)G * (w + h) + sizeof(float2) * (size_t)h * G : 0;
    s.win = 0;
    s.tmp = plane;
    s.tw = s.tmp + (plane > ov ? plane : ov);
    s.scratch = s.tw + sizeof(float2) * (size_t)(w + h);
    s.total = s.scratch + sizeof(Stat6) * (DFT_THREADS / 32);
    return s;
}

// GLOB: the two planes (window / field, and the row transforms / overlap
// tables) of each unit in global scratch, at unit * dftSmem(...).tw bytes,
// for fields whose planes exceed shared memory; the twiddles and the
// reduction scratch stay in shared memory.
template <bool GLOB>
__global__ void __launch_bounds__(DFT_THREADS) k_inverse_dft_t(DhInvParams p, unsigned char* gplanes) {
    extern __shared__ __align__(16) unsigned char dsm[];
    const int unit = blockIdx.x;
    const int pol = unit % p.polCount;
    const int frame = unit / p.polCount;
    const int nx = p.w, ny = p.h;
    const int npix = nx * ny;
    const int ld = nx + 1;
    const int G = p.maxMG > 0 ? p.maxMG : 0;
    const DftSmem L = dftSmem(nx, ny, G);
    unsigned char* pl = GLOB ? gplanes + (size_t)unit * L.tw : dsm;
    const size_t shOff = GLOB ? L.tw : 0;                    // shared memory holds only the twiddles and scratch
    float2* fld = reinterpret_cast<float2*>(pl + L.win);     // window, then the field [ny][ld]
    float2* tmp = reinterpret_cast<float2*>(pl + L.tmp);     // row transforms [ny][ld]; later the overlap tables
    float2* twx = reinterpret_cast<float2*>(dsm + (L.tw - shOff));        // exp(+2 pi i j / nx)
    float2* twy = twx + nx;                                                // exp(+2 pi i j / ny)
    Stat6* scratch = reinterpret_cast<Stat6*>(dsm + (L.scratch - shOff));
    const float2* win = p.window + (size_t)unit * npix;
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int j = e / nx, c = e - j * nx;
        fld[j * ld + c] = win[e];
    }
    for (int j = threadIdx.x; j < nx + ny; j += blockDim.x) {
        const bool isx = j < nx;
        const int k = isx ? j : j - nx, n = isx ? nx : ny;
        double sv, cv;
        sincospi(2.0 * (double)k / (double)n, &sv, &cv);
        twx[j] = make_float2((float)cv, (float)sv);
    }
    __syncthreads();
    // rows: tmp[ky][x] = sum_kx W[ky][kx] exp(+2 pi i kx x / nx)
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int ky = e / nx, x = e - ky * nx;
        const float2* row = fld + ky * ld;
        float ar = 0.f, ai = 0.f;
        int t = 0;
        for (int kx = 0; kx < nx; kx++) {
            const float2 a = row[kx], c = twx[t];
            ar = fmaf(a.x, c.x, fmaf(-a.y, c.y, ar));
            ai = fmaf(a.x, c.y, fmaf(a.y, c.x, ai));
            t += x;
            if (t >= nx) t -= nx;
        }
        tmp[ky * ld + x] = make_float2(ar, ai);
    }
    __syncthreads();
    // columns: fld[y][x] = sum_ky tmp[ky][x] exp(+2 pi i ky y / ny)
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int y = e / nx, x = e - y * nx;
        float ar = 0.f, ai = 0.f;
        int t = 0;
        for (int ky = 0; ky < ny; ky++) {
            const float2 a = tmp[ky * ld + x], c = twy[t];
            ar = fmaf(a.x, c.x, fmaf(-a.y, c.y, ar));
            ai = fmaf(a.x, c.y, fmaf(a.y, c.x, ai));
            t += y;
            if (t >= ny) t -= ny;
        }
        // reference-wave calibration of the IFFT output (digHolo.cpp:8736-8758)
        fld[y * ld + x] = p.refCal ? calMul(make_float2(ar, ai), p.refCal[(size_t)pol * npix + e])
                                   : make_float2(ar, ai);
    }
    __syncthreads();

    // statistics over the untilted field (digHolo.cpp:8866-8870)
    const float inv = (float)(1.0 / ((double)nx * (double)ny));
    const float yShift = fabsf((p.yAxis[1] - p.yAxis[0]) * (float)ny);
    Stat6 st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int y = e / nx, x = e - y * nx;
        const float2 a = fld[y * ld + x];
        const float I0 = fmaf(a.x, a.x, a.y * a.y);
        const float I = I0 * inv;
        const int idx = 2 * y * nx + x;
        if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
        const float yv = p.yAxis[y];
        st.P += I;
        st.cx = fmaf(p.xAxis[x], I, st.cx);
        st.cy = fmaf(yv, I, st.cy);
        st.cyw = fmaf(yv + (yv < 0.f ? yShift : 0.f), I, st.cyw);
        st.e4 = fmaf(I, I, st.e4);
    }
    st = blockReduceStat(st, scratch);
    const float maxAbs = sqrtf(st.maxI);
    const float scale = (float)(32767.0 / (double)maxAbs);
    if (threadIdx.x == 0) {
        const int S = p.statsStride;
        float* s = p.stats;
        const int col = pol * S + frame;
        const int per = p.polCount * S;
        s[0 * per + col] = st.P;
        s[1 * per + col] = st.cx / st.P;
        s[2 * per + col] = st.cy / st.P;
        s[3 * per + col] = scale;
        s[4 * per + col] = __int_as_float(st.maxIdx);
        s[5 * per + col] = p.dA * (st.P * st.P / st.e4);
        s[6 * per + col] = st.cyw / st.P;
    }

    // reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833)
    const short* ref = p.refWave + (size_t)pol * 2 * (nx + ny);
    const float K = (float)(1.0 / (16383.0 * 16383.0));
    const size_t fieldOff = (size_t)unit * npix;
    for (int e = threadIdx.x; e < npix; e += blockDim.x) {
        const int y = e / nx, x = e - y * nx;
        const int xr = ref[x], xi = ref[nx + x];
        const int yr = ref[2 * nx + y], yi = ref[2 * nx + ny + y];
        const float adjR = (float)(yr * xr - yi * xi) * K;
        const float adjI = (float)(yr * xi + yi * xr) * K;
        const float2 a = fld[y * ld + x];
        const float vr = __fsub_rn(__fmul_rn(a.y, adjI), __fmul_rn(a.x, adjR));
        const float vi = __fadd_rn(__fmul_rn(a.x, adjI), __fmul_rn(a.y, adjR));
        if (p.field32) {
            const float* rf = p.refWaveF + (size_t)pol * 2 * (nx + ny);
            const float2 rx = make_float2(rf[x], rf[nx + x]);
            const float2 ry = make_float2(rf[2 * nx + y], rf[2 * nx + ny + y]);
            const float2 v = cmul(a, cmul(ry, rx));
            p.field32[fieldOff + e] = make_float2(-v.x, v.y);
        }
        const short sr = roundSat16(scale * vr);
        const short si = roundSat16(scale * vi);
        p.fieldR[fieldOff + e] = sr;
        p.fieldI[fieldOff + e] = si;
        fld[y * ld + x] = make_float2((float)sr, (float)si);
    }
    if (G <= 0 || !p.coefs) return;   // uniform over the block
    __syncthreads();

    // separable overlap on the int16 field (digHolo.cpp:2149-2341):
    // T[y][m] = sum_x F[y][x] Hx[m][x];  c_mn = sum_y Hy[n][y] T[y][m]
    float* hx = reinterpret_cast<float*>(tmp);   // [G][nx]
    float* hy = hx + G * nx;                     // [G][ny]
    float2* T = reinterpret_cast<float2*>(hy + G * ny);   // [ny][G]
    const short* gx = p.hgX + (size_t)pol * G * nx;
    const short* gy = p.hgY + (size_t)pol * G * ny;
    for (int e = threadIdx.x; e < G * nx; e += blockDim.x) hx[e] = (float)gx[e];
    for (int e = threadIdx.x; e < G * ny; e += blockDim.x) hy[e] = (float)gy[e];
    __syncthreads();
    for (int e = threadIdx.x; e < ny * G; e += blockDim.x) {
        const int m = e / ny, y = e - m * ny;
        const float2* row = fld + y * ld;
        const float* hm = hx + m * nx;
        float ar = 0.f, ai = 0.f;
        for (int x = 0; x < nx; x++) {
            const float2 f = row[x];
            const float hv = hm[x];
            ar = fmaf(f.x, hv, ar);
            ai = fmaf(f.y, hv, ai);
        }
        T[y * G + m] = make_float2(ar, ai);
    }
    __syncthreads();
    const float fieldScale = 1.0f / scale;
    const float* sxp = p.hgScaleX + pol * G;
    const float* syp = p.hgScaleY + pol * G;
    for (int mode = threadIdx.x; mode < p.modeCount; mode += blockDim.x) {
        // mode -> (m, n): group g, n = mode - g(g+1)/2, m = g - n (digHolo.cpp:1245-1265)
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2;
        const int m = g - n;
        const float* hn = hy + n * ny;
        float cr = 0.f, ci = 0.f;
        for (int y = 0; y < ny; y++) {
            const float2 t = T[y * G + m];
            cr = fmaf(hn[y], t.x, cr);
            ci = fmaf(hn[y], t.y, ci);
        }
        const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
        p.coefs[(size_t)frame * p.polCount * p.modeCount + pol * p.modeCount + mode] = make_float2(cr * ms, ci * ms);
    }
}

// Up to four axes per launch (one block each); up to 4 samples per thread.
struct DhBasisJobs {
    DhBasisParams job[4];
};

__global__ void __launch_bounds__(1024) k_basis(DhBasisJobs jobs) {
    const DhBasisParams& p = jobs.job[blockIdx.x];
    __shared__ double red[32];
    __shared__ double sMax;
    const int L = p.count;
    const double W0 = p.w0;
    const double x0 = (double)p.axis[0], xL = (double)p.axis[L - 1];
    const double dX = fabs((xL - x0) / (double)(L - 1));
    const double axisScale = sqrt(2.0) / W0;
    const double step = 4.0 * dX * (sqrt(2.0) / W0);
    const double norm = (1.0 / sqrt(W0)) * sqrt(dX) / sqrt(sqrt(0.5));
    constexpr int PER = 4;
    double u[PER], h0[PER], h1[PER];
    int idx[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int i = threadIdx.x + q * blockDim.x;
        idx[q] = i;
        u[q] = 0.0;
        if (i < L) {
            // u as digHolo forms it: lane value plus (i/4) sequential steps
            double v = axisScale * (double)p.axis[i & 3];
            for (int b = 0; b < (i >> 2); b++) v += step;
            u[q] = v;
        }
        h0[q] = 0.0;
        h1[q] = 0.0;
    }
    for (int mode = 0; mode < p.modes; mode++) {
        double val[PER];
        double localMax = 0.0;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            double v = 0.0;
            if (idx[q] < L) {
                if (mode == 0) v = 0.7511255444649425 * exp(-0.5 * u[q] * u[q]);
                else if (mode == 1) v = 1.0622519320271970 * u[q] * exp(-0.5 * u[q] * u[q]);
                else v = sqrt(2.0 / mode) * u[q] * h1[q] - sqrt((mode - 1.0) / mode) * h0[q];
            }
            h0[q] = h1[q];
            h1[q] = v;
            val[q] = norm * v;
            localMax = fmax(localMax, fabs(val[q]));
        }
        for (int off = 16; off > 0; off >>= 1) localMax = fmax(localMax, __shfl_down_sync(0xffffffffu, localMax, off));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = localMax;
        __syncthreads();
        if (threadIdx.x == 0) {
            double mx = 0.0;
            for (int i = 0; i < (int)(blockDim.x >> 5); i++) mx = fmax(mx, red[i]);
            sMax = mx;
        }
        __syncthreads();
        const double sf = 32767.0 / sMax;
        const float sff = (float)sf;
        const bool q16 = mode < p.modes16;
        if (threadIdx.x == 0 && q16) p.scale[mode] = (float)(1.0 / sf);
#pragma unroll
        for (int q = 0; q < PER; q++) {
            if (idx[q] < L) {
                const float r = rintf(__fmul_rn((float)val[q], sff));
                const int ir = (r >= -2147483648.0f && r < 2147483648.0f) ? (int)r : INT32_MIN;
                if (q16) p.out16[(size_t)mode * L + idx[q]] = (short)max(-32768, min(32767, ir));
                if (p.outF) p.outF[(size_t)mode * L + idx[q]] = (float)val[q];
            }
        }
        __syncthreads();
    }
}

// Transpose of each frame: in is [Ny rows][Nx columns], out[f][i * Ny + j] =
// in[f][j * Nx + i] ([Nx rows][Ny columns]).  32 x 32 tiles through shared
// memory.
__global__ void k_untranspose_u16(const unsigned short* __restrict__ in, unsigned short* __restrict__ out, int Nx,
                                  int Ny, int frames) {
    __shared__ unsigned short tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const size_t fp = (size_t)Nx * Ny;
    for (int f = blockIdx.z; f < frames; f += gridDim.z) {
        const unsigned short* src = in + (size_t)f * fp;
        unsigned short* dst = out + (size_t)f * fp;
        for (int k = 0; k < 32; k += 8) {
            const int j = j0 + ty + k, i = i0 + tx;
            if (j < Ny && i < Nx) tile[ty + k][tx] = src[(size_t)j * Nx + i];
        }
        __syncthreads();
        for (int k = 0; k < 32; k += 8) {
            const int i = i0 + ty + k, j = j0 + tx;
            if (i < Nx && j < Ny) dst[(size_t)i * Ny + j] = tile[tx][ty + k];
        }
        __syncthreads();
    }
}

cudaError_t dh_launch_untranspose_u16(const unsigned short* in, unsigned short* out, int Nx, int Ny, int frames,
                                      cudaStream_t s) {
    if (frames <= 0) return cudaSuccess;
    dim3 grid((Nx + 31) / 32, (Ny + 31) / 32, frames < 65535 ? frames : 65535);
    k_untranspose_u16<<<grid, dim3(32, 8), 0, s>>>(in, out, Nx, Ny, frames);
    return cudaGetLastError();
}

// int16 field -> complex64 x (1/scale) (digHolo.cpp:4947-4981).
__global__ void k_fields_to_c64(const short* R, const short* I, const float* stats, int statsStride,
                                int polCount, int frameCount, int npix, float2* out) {
    const size_t total = (size_t)frameCount * polCount * npix;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t unit = e / npix;
        const int pol = (int)(unit % polCount);
        const int frame = (int)(unit / polCount);
        const float scale = stats[3 * polCount * statsStride + pol * statsStride + frame];
        const float inv = (float)(1.0 / (double)scale);
        out[e] = make_float2((float)R[e] * inv, (float)I[e] * inv);
    }
}

// ------------------------------------------------------------------ launchers

size_t dh_forward_smem_bytes(int logW, int logH, int colChunk) {
    const int N = 1 << (logW - 1);
    int RB = FWD_ROWBUF_ELEMS / N;
    if (RB > (1 << logH)) RB = 1 << logH;
    return sizeof(float2) * ((size_t)RB * N + (size_t)(1 << logH) * colChunk);
}

cudaError_t dh_launch_forward(const DhFwdParams& p, cudaStream_t s) {
    const size_t smem = dh_forward_smem_bytes(p.logW, p.logH, p.colChunk);
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_forward), (int)smem);
    if (e != cudaSuccess) return e;
    const long long blocks = (long long)p.frameCount * p.polCount * (p.w / p.colChunk);
    k_forward<<<(unsigned)blocks, FWD_THREADS, smem, s>>>(p);
    return cudaGetLastError();
}

size_t dh_inverse_smem_bytes(const DhInvParams& p) {
    const int nx = p.lowres ? (1 << p.logw) : (1 << p.logW);
    const int ny = p.lowres ? (1 << p.logh) : (1 << p.logH);
    size_t bytes = sizeof(float2) * (size_t)(nx + 1) * ny;
    if (!p.lowres) bytes += sizeof(float2) * (size_t)(1 << p.logH) * (1 << p.logw);
    size_t extra = sizeof(Stat6) * (INV_THREADS / 32);
    if (p.maxMG > 0) {
        const size_t ov = sizeof(float) * (size_t)p.maxMG * (nx + ny) + sizeof(float2) * (size_t)ny * p.maxMG;
        if (ov > extra) extra = ov;
    }
    return bytes + extra;
}

cudaError_t dh_launch_inverse(const DhInvParams& p, cudaStream_t s) {
    if (p.w != (1 << p.logw) || p.h != (1 << p.logh)) return cudaErrorNotSupported;   // power-of-two windows only
    const size_t smem = dh_inverse_smem_bytes(p);
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_inverse), (int)smem);
    if (e != cudaSuccess) return e;
    // small (low-resolution) fields: one thread per pair of pixels, at least two warps
    int threads = INV_THREADS;
    if (p.lowres) {
        const int npix = (1 << p.logw) * (1 << p.logh);
        threads = npix / 2;
        if (threads < 64) threads = 64;
        if (threads > INV_THREADS) threads = INV_THREADS;
    }
    k_inverse<<<(unsigned)(p.frameCount * p.polCount), threads, smem, s>>>(p);
    return cudaGetLastError();
}

// Shared memory of the low-resolution DFT kernel for w x h fields and maxMG G.
size_t dh_inverse_dft_smem_bytes(int w, int h, int G) { return dftSmem(w, h, G > 0 ? G : 0).total; }

// Low-resolution fields whose sides are multiples of 16 (any, including the
// powers of two); cudaErrorNotSupported when the field does not fit shared memory.
cudaError_t dh_launch_inverse_dft(const DhInvParams& p, cudaStream_t s) {
    if (!p.lowres || p.w < 16 || p.h < 16 || p.w % 16 || p.h % 16) return cudaErrorNotSupported;
    const size_t smem = dh_inverse_dft_smem_bytes(p.w, p.h, p.maxMG);
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_inverse_dft_t<false>), (int)smem);
    if (e != cudaSuccess) return e;
    if (p.frameCount * p.polCount <= 0) return cudaSuccess;
    k_inverse_dft_t<false><<<(unsigned)(p.frameCount * p.polCount), DFT_THREADS, smem, s>>>(p, nullptr);
    return cudaGetLastError();
}

// Scratch of the global-plane variant: each unit's two planes.
size_t dh_inverse_dft_global_bytes(const DhInvParams& p) {
    if (!p.lowres || p.w < 16 || p.h < 16 || p.w % 16 || p.h % 16) return 0;
    return dftSmem(p.w, p.h, p.maxMG > 0 ? p.maxMG : 0).tw * (size_t)(p.frameCount * p.polCount);
}

// Low-resolution fields of any multiple of 16 whose planes exceed shared
// memory: the same kernel with the planes in global scratch
// (dh_inverse_dft_global_bytes); cudaErrorNotSupported outside its shapes.
cudaError_t dh_launch_inverse_dft_global(const DhInvParams& p, void* scratch, size_t scratchBytes, cudaStream_t s) {
    if (!p.lowres || p.w < 16 || p.h < 16 || p.w % 16 || p.h % 16 || p.w > 4096 || p.h > 4096)
        return cudaErrorNotSupported;
    if (p.frameCount * p.polCount <= 0) return cudaSuccess;
    const DftSmem L = dftSmem(p.w, p.h, p.maxMG > 0 ? p.maxMG : 0);
    if (!scratch || scratchBytes < L.tw * (size_t)(p.frameCount * p.polCount) ||
        (reinterpret_cast<uintptr_t>(scratch) & 15))
        return cudaErrorInvalidValue;
    const size_t smem = L.total - L.tw;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_inverse_dft_t<true>), (int)smem);
    if (e != cudaSuccess) return e;
    k_inverse_dft_t<true><<<(unsigned)(p.frameCount * p.polCount), DFT_THREADS, smem, s>>>(
        p, static_cast<unsigned char*>(scratch));
    return cudaGetLastError();
}

// n <= 4 axes in one launch.
cudaError_t dh_launch_basis_jobs(const DhBasisParams* ps, int n, cudaStream_t s) {
    if (n < 1 || n > 4) return cudaErrorInvalidValue;
    DhBasisJobs jobs;
    memset(&jobs, 0, sizeof(jobs));
    int threads = 32;
    for (int i = 0; i < n; i++) {
        jobs.job[i] = ps[i];
        int t = (ps[i].count + 3) / 4;
        t = ((t + 31) / 32) * 32;
        threads = t > threads ? t : threads;
    }
    if (threads > 1024) return cudaErrorInvalidValue;
    k_basis<<<n, threads, 0, s>>>(jobs);
    return cudaGetLastError();
}

cudaError_t dh_launch_basis(const DhBasisParams& p, cudaStream_t s) { return dh_launch_basis_jobs(&p, 1, s); }

cudaError_t dh_launch_fields_to_c64(const short* R, const short* I, const float* stats, int statsStride,
                                    int polCount, int frameCount, int npix, float2* out, cudaStream_t s) {
    const size_t total = (size_t)frameCount * polCount * npix;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    k_fields_to_c64<<<blocks, 256, 0, s>>>(R, I, stats, statsStride, polCount, frameCount, npix, out);
    return cudaGetLastError();
}

// Sum over the batch of |E|^2 / (nx ny) per pixel, from the int16 fields
// (the batch-sum intensity of digHoloFieldAnalysis, digHolo.cpp:2519-2568).
__global__ void k_batchsum(const short* R, const short* I, const float* stats, int statsStride,
                           int polCount, int frameCount, int npix, float* out) {
    const float inv = 1.0f / (float)npix;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < polCount * npix; e += gridDim.x * blockDim.x) {
        const int pol = e / npix, pix = e - pol * npix;
        float acc = 0.f;
        for (int f = 0; f < frameCount; f++) {
            const float scale = stats[3 * polCount * statsStride + pol * statsStride + f];
            const float s = (float)(1.0 / (double)scale);
            const size_t o = ((size_t)f * polCount + pol) * npix + pix;
            const float r = (float)R[o] * s, i = (float)I[o] * s;
            acc += (r * r + i * i) * inv;
        }
        out[e] = acc;
    }
}

cudaError_t dh_launch_batchsum(const short* R, const short* I, const float* stats, int statsStride,
                               int polCount, int frameCount, int npix, float* out, cudaStream_t s) {
    int blocks = (polCount * npix + 255) / 256;
    if (blocks < 1) blocks = 1;
    k_batchsum<<<blocks, 256, 0, s>>>(R, I, stats, statsStride, polCount, frameCount, npix, out);
    return cudaGetLastError();
}

// Frame averaging of the Fourier windows: the two-pass branch of
// digHoloCopyWindow (digHolo.cpp:1886-1932, 2062-2118) as driven per batch
// item by digHolo.cpp:8636-8672.  One block per (batch item, polarisation)
// over the windows of all batch x avg frames: the first frame's window
// x 1/avg; each further window x the unit phase of sum(acc conj(window))
// x 1/avg, added.  Frames of batch item b: b avg + k (sequential, mode 0),
// k batch + b (interlaced, mode 1), b + k (sweeps of one wavelength, mode 2).
// The batch calibration factor of item b multiplies every window of it in
// the reference; the alignment phase is blind to a common factor, so it is
// applied once to the average.  Each thread owns the same pixels in every
// pass, so only the correlation needs the block.
__global__ void __launch_bounds__(256) k_average_windows(const float2* __restrict__ in, float2* __restrict__ out,
                                                         int batch, int avg, int mode, int polCount, int n,
                                                         const float2* __restrict__ cal, int calCount) {
    __shared__ double red[2][8];
    const int b = blockIdx.x / polCount, pol = blockIdx.x - b * polCount;
    float2* acc = out + ((size_t)b * polCount + pol) * n;
    const float inv = (float)(1.0 / avg);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (int k = 0; k < avg; k++) {
        const int f = mode == 0 ? b * avg + k : (mode == 1 ? k * batch + b : b + k);
        const float2* src = in + ((size_t)f * polCount + pol) * n;
        if (k == 0) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const float2 v = src[i];
                acc[i] = make_float2(v.x * inv, v.y * inv);
            }
            continue;
        }
        double cr = 0, ci = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float2 a = acc[i], v = src[i];
            cr += (double)a.x * v.x + (double)a.y * v.y;
            ci += (double)a.y * v.x - (double)a.x * v.y;
        }
        for (int off = 16; off > 0; off >>= 1) {
            cr += __shfl_xor_sync(0xffffffffu, cr, off);
            ci += __shfl_xor_sync(0xffffffffu, ci, off);
        }
        __syncthreads();   // the previous pass has read red
        if (lane == 0) { red[0][warp] = cr; red[1][warp] = ci; }
        __syncthreads();
        cr = 0; ci = 0;
        for (int w = 0; w < warps; w++) { cr += red[0][w]; ci += red[1][w]; }
        const double m = sqrt(cr * cr + ci * ci);
        const float pr = (float)(cr / m) * inv, pi = (float)(ci / m) * inv;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float2 a = acc[i], v = src[i];
            acc[i] = make_float2(a.x + (v.x * pr - v.y * pi), a.y + (v.x * pi + v.y * pr));
        }
    }
    if (cal && calCount > 0) {
        const float2 c = cal[pol * calCount + (b % calCount)];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float2 a = acc[i];
            acc[i] = make_float2(a.x * c.x - a.y * c.y, a.x * c.y + a.y * c.x);
        }
    }
}

cudaError_t dh_launch_average_windows(const float2* in, float2* out, int batch, int avg, int mode, int polCount,
                                      int n, const float2* cal, int calCount, cudaStream_t s) {
    if (batch <= 0 || polCount <= 0 || n <= 0) return cudaSuccess;
    if (avg < 1 || mode < 0 || mode > 2) return cudaErrorInvalidValue;
    k_average_windows<<<batch * polCount, 256, 0, s>>>(in, out, batch, avg, mode, polCount, n, cal, calCount);
    return cudaGetLastError();
}

// Coefficients in another basis (digHoloApplyBasisTransform,
// digHolo.cpp:9469-9600): per (batch item, polarisation) out[j] =
// sum_{i < din} T[i][j] in[i] for j < dout, T [din][dout] complex, no
// conjugation (the reference's cgemv, no transpose, of the column-major
// [dout x din] matrix).  One block per row; the input row staged in shared
// memory, consecutive threads on consecutive outputs.
__global__ void __launch_bounds__(128) k_basis_transform(const float2* __restrict__ in, float2* __restrict__ out,
                                                         const float2* __restrict__ T, int M, int din, int dout) {
    extern __shared__ float2 xrow[];
    const int row = blockIdx.x;   // batch item x polarisation
    const float2* x = in + (size_t)row * M;
    for (int i = threadIdx.x; i < din; i += blockDim.x) xrow[i] = x[i];
    __syncthreads();
    for (int j = threadIdx.x; j < dout; j += blockDim.x) {
        float ar = 0.f, ai = 0.f;
        for (int i = 0; i < din; i++) {
            const float2 t = T[(size_t)i * dout + j], v = xrow[i];
            ar = fmaf(v.x, t.x, fmaf(-v.y, t.y, ar));
            ai = fmaf(v.x, t.y, fmaf(v.y, t.x, ai));
        }
        out[(size_t)row * dout + j] = make_float2(ar, ai);
    }
}

cudaError_t dh_launch_basis_transform(const float2* in, float2* out, const float2* T, int rows, int M, int din, int dout,
                                      cudaStream_t s) {
    if (rows <= 0 || dout <= 0) return cudaSuccess;
    if (din < 1 || din > M) return cudaErrorInvalidValue;
    const size_t smem = sizeof(float2) * (size_t)din;
    if (smem > 48 * 1024) {
        cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_basis_transform), (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_basis_transform<<<(unsigned)rows, 128, smem, s>>>(in, out, T, M, din, dout);
    return cudaGetLastError();
}
