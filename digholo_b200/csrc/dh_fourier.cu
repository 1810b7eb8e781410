// Full R2C Fourier planes of the FFT windows and their analysis: the
// reference's digHoloPixelsFourierPlane (FFTW r2c, digHolo.cpp:7184-7260)
// and digHoloFFTAnalysis (digHolo.cpp:6931-6980 -> 8990-9180 -> 2354-2654).
// The batch path never forms these planes (its forward transform is pruned
// to the IFFT window); they are computed on request from the batch's frames.
//
// Plane: rows by a packed half-length complex FFT plus the R2C split, then
// columns, both radix-2 in shared memory, FP32.  Analysis, with the
// reference's choices: the plane's column i and row j carry the fftshifted
// axis values kx[i], ky[j]; pixel (j, i) enters when j is neither 0 nor H/2,
// 0 < i < 8 floor(Nx/8) (Nx = W/2+1), and kx[i]^2 + ky[j]^2 >= R^2 (the
// DC disk, R = 2 k0 sin(aperture)); intensity I = |F|^2/(Nx H).  The
// per-frame maximum is of |F|^2, the batch entry's of the summed normalised
// intensity, whose index the reference reports 8 positions on.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"

using namespace dh;

bool dh_plane_window64_fits(const DhFourierParams& q);
cudaError_t dh_launch_plane_rows512(const DhFourierParams& q, int compact, cudaStream_t s);
cudaError_t dh_launch_plane_window64(const DhFourierParams& q, cudaStream_t s);


namespace {

constexpr int FT = 256;           // threads per block
constexpr int FBUF = 4096;        // complex elements per shared transform buffer

// RB rows of one (frame, polarisation) window: packed FFT of length W/2, R2C
// split, all W/2+1 columns written.
__global__ void __launch_bounds__(FT) k_fourier_rows(DhFourierParams q) {
    extern __shared__ float2 sm[];
    const DhFwdParams& f = q.f;
    const int W = 1 << f.logW, H = 1 << f.logH, N = W / 2, logN = f.logW - 1;
    const int Nx = N + 1;
    int RB = FBUF / N;
    if (RB > H) RB = H;
    const int groups = H / RB;
    const int unit = blockIdx.x / groups, r0 = (blockIdx.x % groups) * RB;
    const int P = f.polCount, pol = unit % P, frame = unit / P;
    const long long base = (long long)frame * f.frameStride + (long long)f.cy[pol] * f.frameWidth + f.cx[pol];
    // pixel pairs (2n, 2n + 1) in one load: the window's corner and the row
    // pitch are even, and the frame buffers are 16-byte aligned
    for (int e = threadIdx.x; e < RB * N; e += FT) {
        const int r = e / N, n = e - r * N;
        const long long o = base + (long long)(r0 + r) * f.frameWidth + 2 * n;
        float2 v;
        if (f.inputU16) {
            const unsigned int u = *reinterpret_cast<const unsigned int*>(static_cast<const unsigned short*>(f.frames) + o);
            v = make_float2((float)(u & 0xFFFFu), (float)(u >> 16));
        } else {
            v = *reinterpret_cast<const float2*>(static_cast<const float*>(f.frames) + o);
        }
        sm[r * N + bitrev(n, logN)] = v;
    }
    __syncthreads();
    fft_dit(sm, RB, N, 1, logN, false, false, f.twiddle);
    float2* out = q.plane + ((size_t)unit * H + r0) * Nx;
    // all W/2 + 1 columns, or with windowCols the Fourier window's w columns
    const int kcount = q.windowCols ? f.w : Nx;
    const int kbeg = q.windowCols ? f.sx0[pol] : 0;
    for (int e = threadIdx.x; e < RB * kcount; e += FT) {
        const int r = e / kcount, k = kbeg + (e - r * kcount);
        const float2 zk = sm[r * N + (k & (N - 1))];
        const float2 zc = cconj(sm[r * N + ((N - k) & (N - 1))]);
        const float2 even = cscale(cadd(zk, zc), 0.5f);
        const float2 d = csub(zk, zc);
        const float2 odd = make_float2(0.5f * d.y, -0.5f * d.x);   // -i/2 (zk - zc)
        const float2 wk = __ldg(&f.twiddle[k << (TW_LOG - f.logW)]);
        out[(size_t)r * Nx + k] = cadd(even, cmul(wk, odd));
    }
}

// CB columns of one plane: H-point forward FFT in place.  With windowCols
// only the columns sx0 .. sx0 + w - 1 of the unit's polarisation (the
// Fourier window's) are transformed; the others are left as the rows wrote them.
__global__ void __launch_bounds__(FT) k_fourier_cols(DhFourierParams q) {
    extern __shared__ float2 sm[];
    const DhFwdParams& f = q.f;
    const int W = 1 << f.logW, H = 1 << f.logH, Nx = W / 2 + 1;
    int CB = FBUF / H;
    if (CB < 1) CB = 1;
    const int ccount = q.windowCols ? f.w : Nx;
    const int groups = (ccount + CB - 1) / CB;
    const int unit = blockIdx.x / groups;
    const int cbeg = q.windowCols ? f.sx0[unit % f.polCount] : 0;
    const int c0 = cbeg + (blockIdx.x % groups) * CB;
    const int cols = cbeg + ccount - c0 < CB ? cbeg + ccount - c0 : CB;
    float2* pl = q.plane + (size_t)unit * H * Nx;
    for (int e = threadIdx.x; e < H * cols; e += FT) {
        const int r = e / cols, c = e - r * cols;
        sm[bitrev(r, f.logH) * cols + c] = pl[(size_t)r * Nx + c0 + c];
    }
    __syncthreads();
    fft_dit(sm, cols, 1, cols, f.logH, false, true, f.twiddle);
    for (int e = threadIdx.x; e < H * cols; e += FT) {
        const int r = e / cols, c = e - r * cols;
        pl[(size_t)r * Nx + c0 + c] = sm[r * cols + c];
    }
}

struct FStat {
    float maxV;
    int maxIdx;
    float P, cx, cy, cyw, e4;
};

__device__ __forceinline__ void fMerge(FStat& a, const FStat& b) {
    if (b.maxV > a.maxV || (b.maxV == a.maxV && b.maxIdx > a.maxIdx)) { a.maxV = b.maxV; a.maxIdx = b.maxIdx; }
    a.P += b.P; a.cx += b.cx; a.cy += b.cy; a.cyw += b.cyw; a.e4 += b.e4;
}

__device__ __forceinline__ bool inside(const DhFourierParams& q, int j, int i, int H, int Nx) {
    const int nxr = 8 * (Nx / 8);
    if (j == 0 || j == H / 2 || i == 0 || i >= nxr) return false;
    if (q.r2 == 0.f) return true;
    const float x = q.kx[i], y = q.ky[j];
    return __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)) >= q.r2;
}

// Block reduction of the statistics and their store into column `col`.
__device__ void finishStats(const DhFourierParams& q, FStat st, int pol, int col, int idxOffset) {
    __shared__ FStat red[FT / 32];
    for (int off = 16; off > 0; off >>= 1) {
        FStat o;
        o.maxV = __shfl_xor_sync(0xffffffffu, st.maxV, off);
        o.maxIdx = __shfl_xor_sync(0xffffffffu, st.maxIdx, off);
        o.P = __shfl_xor_sync(0xffffffffu, st.P, off);
        o.cx = __shfl_xor_sync(0xffffffffu, st.cx, off);
        o.cy = __shfl_xor_sync(0xffffffffu, st.cy, off);
        o.cyw = __shfl_xor_sync(0xffffffffu, st.cyw, off);
        o.e4 = __shfl_xor_sync(0xffffffffu, st.e4, off);
        fMerge(st, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = st;
    __syncthreads();
    if (threadIdx.x != 0) return;
    FStat t = red[0];
    for (int w = 1; w < FT / 32; w++) fMerge(t, red[w]);
    const float dA = fabsf(q.kx[2] - q.kx[1]) * fabsf(q.ky[2] - q.ky[1]);
    const int P = q.f.polCount, S = q.f.frameCount + 1;
    float* s = q.stats;
    const int c = pol * S + col, per = P * S;
    s[0 * per + c] = t.P;
    s[1 * per + c] = t.cx / t.P;
    s[2 * per + c] = t.cy / t.P;
    s[3 * per + c] = (float)(32767.0 / (double)sqrtf(t.maxV));
    s[4 * per + c] = __int_as_float(t.maxIdx + idxOffset);
    s[5 * per + c] = dA * (t.P * t.P / t.e4);
    s[6 * per + c] = t.cyw / t.P;
}

// Per (frame, polarisation) statistics of the plane.
__global__ void __launch_bounds__(FT) k_fourier_stats(DhFourierParams q) {
    const int W = 1 << q.f.logW, H = 1 << q.f.logH, Nx = W / 2 + 1;
    const int unit = blockIdx.x, P = q.f.polCount, pol = unit % P, frame = unit / P;
    const float norm = (float)(1.0 / ((double)Nx * (double)H));
    const float yShift = fabsf((q.ky[1] - q.ky[0]) * (float)H);
    const float2* pl = q.plane + (size_t)unit * H * Nx;
    FStat st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int e = threadIdx.x; e < H * Nx; e += FT) {
        const int j = e / Nx, i = e - j * Nx;
        if (!inside(q, j, i, H, Nx)) continue;
        const float2 v = pl[e];
        const float I0 = fmaf(v.x, v.x, v.y * v.y);
        const float I = I0 * norm;
        const int idx = 2 * j * Nx + i;
        if (I0 > st.maxV || (I0 == st.maxV && idx > st.maxIdx)) { st.maxV = I0; st.maxIdx = idx; }
        const float y = q.ky[j];
        st.P += I;
        st.cx = fmaf(q.kx[i], I, st.cx);
        st.cy = fmaf(y, I, st.cy);
        st.cyw = fmaf(y + (y < 0.f ? yShift : 0.f), I, st.cyw);
        st.e4 = fmaf(I, I, st.e4);
    }
    finishStats(q, st, pol, frame, 0);
}

// Batch-sum intensity per pixel (zero outside the analysed region).
__global__ void k_fourier_batchsum(DhFourierParams q) {
    const int W = 1 << q.f.logW, H = 1 << q.f.logH, Nx = W / 2 + 1;
    const int P = q.f.polCount, B = q.f.frameCount;
    const float norm = (float)(1.0 / ((double)Nx * (double)H));
    const int total = P * H * Nx;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int pol = e / (H * Nx), pix = e - pol * H * Nx;
        const int j = pix / Nx, i = pix - j * Nx;
        float acc = 0.f;
        if (inside(q, j, i, H, Nx)) {
            for (int b = 0; b < B; b++) {
                const float2 v = q.plane[((size_t)b * P + pol) * H * Nx + pix];
                acc += fmaf(v.x, v.x, v.y * v.y) * norm;
            }
        }
        q.batchSum[(size_t)pol * W * H + pix] = acc;
    }
}

// Statistics of the batch-sum intensity (the frameCount column).
__global__ void __launch_bounds__(FT) k_fourier_sum_stats(DhFourierParams q) {
    const int W = 1 << q.f.logW, H = 1 << q.f.logH, Nx = W / 2 + 1;
    const int pol = blockIdx.x;
    const float yShift = fabsf((q.ky[1] - q.ky[0]) * (float)H);
    const float* S = q.batchSum + (size_t)pol * W * H;
    FStat st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int e = threadIdx.x; e < H * Nx; e += FT) {
        const int j = e / Nx, i = e - j * Nx;
        if (!inside(q, j, i, H, Nx)) continue;
        const float I = S[e];
        const int idx = 2 * j * Nx + i;
        if (I > st.maxV || (I == st.maxV && idx > st.maxIdx)) { st.maxV = I; st.maxIdx = idx; }
        const float y = q.ky[j];
        st.P += I;
        st.cx = fmaf(q.kx[i], I, st.cx);
        st.cy = fmaf(y, I, st.cy);
        st.cyw = fmaf(y + (y < 0.f ? yShift : 0.f), I, st.cyw);
        st.e4 = fmaf(I, I, st.e4);
    }
    finishStats(q, st, pol, q.f.frameCount, 8);
}

}  // namespace

// Fourier window of each (frame, polarisation) from its full plane: rows
// (j + SY + H/2) mod H, columns sx0 .. sx0 + w - 1 of the R2C plane, times the
// batch calibration and the window factors (mask, normalisation, inverse
// pixel sinc, beam-centre phase: tabAdj), as digHoloCopyWindow
// (digHolo.cpp:1808-2122) and the pruned forward kernels.
__global__ void k_window_from_plane(DhFourierParams q) {
    const DhFwdParams& f = q.f;
    const int W = 1 << f.logW, H = 1 << f.logH, Nx = W / 2 + 1;
    const int P = f.polCount, w = f.w, h = f.h;
    const int total = f.frameCount * P * h * w;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int c = e % w, j = (e / w) % h, unit = e / (w * h);
        const int pol = unit % P, frame = unit / P;
        const int row = (j + f.sy[pol] + H / 2) & (H - 1);
        float2 Y = q.plane[((size_t)unit * H + row) * Nx + f.sx0[pol] + c];
        if (f.batchCal && f.batchCalCount > 0)
            Y = cmul(Y, f.batchCal[pol * f.batchCalCount + ((f.frameOffset + frame) % f.batchCalCount)]);
        f.window[e] = cmul(Y, f.tabAdj[((size_t)pol * h + j) * w + c]);
    }
}

// Forward stage through the full planes (windows of 256 pixels or more,
// where the pruned kernels do not apply): q.plane receives the R2C planes,
// q.f.window the Fourier windows.  cudaErrorNotSupported when a window
// column falls outside the R2C half plane or the tables are missing.
cudaError_t dh_launch_forward_plane(const DhFourierParams& q, cudaStream_t s) {
    const DhFwdParams& f = q.f;
    const int W = 1 << f.logW, H = 1 << f.logH, N = W / 2;
    if (!f.tabAdj || !q.plane || W < 16 || H < 16 || W > TW_N || H > TW_N) return cudaErrorNotSupported;
    for (int p = 0; p < f.polCount; p++)
        if (f.sx0[p] < 0 || f.sx0[p] + f.w > N + 1) return cudaErrorNotSupported;
    const int units = f.frameCount * f.polCount;
    if (units <= 0) return cudaSuccess;
    int RB = FBUF / N;
    if (RB > H) RB = H;
    int CB = FBUF / H;
    if (CB < 1) CB = 1;
    const int Nx = N + 1;
    const size_t smemR = sizeof(float2) * (size_t)RB * N, smemC = sizeof(float2) * (size_t)H * CB;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_fourier_rows), (int)smemR);
    if (e != cudaSuccess) return e;
    e = setSmemOnce(reinterpret_cast<const void*>(k_fourier_cols), (int)smemC);
    if (e != cudaSuccess) return e;
    // the window needs only its own w columns of each plane transformed
    DhFourierParams qw = q;
    qw.windowCols = 1;
    (void)Nx;
    // 512-pixel rows: the register row kernel; with 64-row windows its
    // compact output feeds the pruned column kernel (dh_plane.cu)
    const bool fits64 = dh_plane_window64_fits(qw);
    e = dh_launch_plane_rows512(qw, fits64 ? 1 : 0, s);
    if (e == cudaSuccess) {
        if (fits64) return dh_launch_plane_window64(qw, s);
    } else if (e != cudaErrorNotSupported) {
        return e;
    } else {
        cudaGetLastError();
        k_fourier_rows<<<(unsigned)(units * (H / RB)), FT, smemR, s>>>(qw);
    }
    k_fourier_cols<<<(unsigned)(units * ((f.w + CB - 1) / CB)), FT, smemC, s>>>(qw);
    const int total = units * f.h * f.w;
    int g = (total + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_window_from_plane<<<g, 256, 0, s>>>(qw);
    return cudaGetLastError();
}

// Fourier planes and their analysis for q.f.frameCount frames.
// cudaErrorNotSupported for window sides above 4096 or under 16.
cudaError_t dh_launch_fourier_full(const DhFourierParams& q, cudaStream_t s) {
    const int W = 1 << q.f.logW, H = 1 << q.f.logH, N = W / 2, Nx = N + 1;
    if (W < 16 || H < 16 || W > TW_N || H > TW_N) return cudaErrorNotSupported;
    const int units = q.f.frameCount * q.f.polCount;
    if (units <= 0) return cudaSuccess;
    int RB = FBUF / N;
    if (RB > H) RB = H;
    if (RB < 1) return cudaErrorNotSupported;
    int CB = FBUF / H;
    if (CB < 1) CB = 1;
    const size_t smemR = sizeof(float2) * (size_t)RB * N, smemC = sizeof(float2) * (size_t)H * CB;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_fourier_rows), (int)smemR);
    if (e != cudaSuccess) return e;
    e = setSmemOnce(reinterpret_cast<const void*>(k_fourier_cols), (int)smemC);
    if (e != cudaSuccess) return e;
    DhFourierParams qf = q;
    qf.windowCols = 0;   // the whole plane
    k_fourier_rows<<<(unsigned)(units * (H / RB)), FT, smemR, s>>>(qf);
    k_fourier_cols<<<(unsigned)(units * ((Nx + CB - 1) / CB)), FT, smemC, s>>>(qf);
    k_fourier_stats<<<(unsigned)units, FT, 0, s>>>(qf);
    const int total = q.f.polCount * H * Nx;
    int g = (total + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    k_fourier_batchsum<<<g, 256, 0, s>>>(q);
    k_fourier_sum_stats<<<(unsigned)q.f.polCount, FT, 0, s>>>(q);
    return cudaGetLastError();
}
