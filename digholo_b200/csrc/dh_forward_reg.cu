// Forward stage, register-resident variant for FFT windows up to 128 pixels
// wide: one thread transforms one window row entirely in registers (packed
// half-length complex FFT, compile-time twiddles from constant memory, no
// barriers inside the transform), and the column transform is evaluated only
// for the IFFT window's rows, as h-point FFTs of the H/h decimated column
// sequences followed by an H/h-term twiddled sum.
//
// Same results as k_forward (dh_kernels.cu) and the reference's
// FFTW r2c + digHoloCopyWindow (digHolo.cpp:7184-7260, 1808-2122).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_params.h"

using namespace dh;

// exp(-2 pi i k / 4096), k < 4096, set once by dh_forward_reg_init.
__constant__ float2 c_tw[TW_N];

namespace {

// In-place radix-2 decimation-in-frequency FFT of N values held in
// registers: natural-order input, bit-reversed output.  Every index is a
// compile-time constant, so the twiddles are constant-bank operands and the
// trivial ones (1, -i) cost nothing.
template <int N>
__device__ __forceinline__ void fftRegDIF(float2 (&v)[N]) {
#pragma unroll
    for (int m = N / 2; m >= 1; m >>= 1) {
#pragma unroll
        for (int blk = 0; blk < N; blk += 2 * m) {
#pragma unroll
            for (int j = 0; j < m; j++) {
                const float2 a = v[blk + j];
                const float2 b = v[blk + j + m];
                v[blk + j] = cadd(a, b);
                const float2 d = csub(a, b);
                // twiddle exp(-2 pi i j / (2m))
                if (j == 0) {
                    v[blk + j + m] = d;
                } else if (2 * j == m) {
                    v[blk + j + m] = make_float2(d.y, -d.x);  // multiply by -i
                } else {
                    const float2 w = c_tw[j * (TW_N / (2 * m))];
                    v[blk + j + m] = cmul(d, w);
                }
            }
        }
    }
}

template <int LOG>
__host__ __device__ constexpr int brevC(int i) {
    int r = 0;
    for (int b = 0; b < LOG; b++) r |= ((i >> b) & 1) << (LOG - 1 - b);
    return r;
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

__device__ __forceinline__ int wrapModF(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

}  // namespace

// Template N: half the FFT-window width (complex samples per row).
// Template HW: IFFT-window height h (rows kept; also the inner FFT length).
// blockDim.x = max(H, w * H / HW); one block per (frame, polarisation).
template <int N, int HW>
__global__ void __launch_bounds__(256) k_forward_reg(DhFwdParams p) {
    constexpr int LOGN = ilog2c(N);
    constexpr int LOGHW = ilog2c(HW);
    constexpr int ZLD = N + 1;  // padded row stride of the Z buffer (complex)
    extern __shared__ float2 sm[];
    const int H = 1 << p.logH;
    const int W = 2 * N;
    const int w = p.w;
    const int Q = H / HW;  // decimation of the column transform
    const int unit = blockIdx.x;
    const int pol = unit % p.polCount;
    const int frame = unit / p.polCount;
    float2* zbuf = sm;                       // H x ZLD
    float2* colbuf = sm + (size_t)H * ZLD;   // H x w
    float2* exch = sm;                       // w x Q x HW (reuses zbuf after the row pass)

    // ---- rows: each thread loads one row and transforms it in registers
    const int tid = threadIdx.x;
    if (tid < H) {
        const long long base = (long long)frame * p.frameStride + (long long)(p.cy[pol] + tid) * p.frameWidth + p.cx[pol];
        float2 v[N];
        if (p.inputU16) {
            const uint4* src = reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(p.frames) + base);
#pragma unroll
            for (int q = 0; q < W / 8; q++) {
                const uint4 u = __ldg(src + q);
                v[4 * q + 0] = make_float2((float)(u.x & 0xFFFFu), (float)(u.x >> 16));
                v[4 * q + 1] = make_float2((float)(u.y & 0xFFFFu), (float)(u.y >> 16));
                v[4 * q + 2] = make_float2((float)(u.z & 0xFFFFu), (float)(u.z >> 16));
                v[4 * q + 3] = make_float2((float)(u.w & 0xFFFFu), (float)(u.w >> 16));
            }
        } else {
            const float4* src = reinterpret_cast<const float4*>(static_cast<const float*>(p.frames) + base);
#pragma unroll
            for (int q = 0; q < W / 4; q++) {
                const float4 f = __ldg(src + q);
                v[2 * q + 0] = make_float2(f.x, f.y);
                v[2 * q + 1] = make_float2(f.z, f.w);
            }
        }
        fftRegDIF<N>(v);
        float2* zr = zbuf + (size_t)tid * ZLD;
#pragma unroll
        for (int i = 0; i < N; i++) zr[brevC<LOGN>(i)] = v[i];
    }
    __syncthreads();

    // ---- R2C split: X[k] for the w kept columns k = sx0 + c
    const int sx0 = p.sx0[pol];
    for (int e = tid; e < H * w; e += blockDim.x) {
        const int r = e / w, c = e - r * w;
        const int k = sx0 + c;
        const float2* zr = zbuf + (size_t)r * ZLD;
        const float2 zk = zr[k & (N - 1)];
        const float2 zc = cconj(zr[(N - k) & (N - 1)]);
        const float2 even = cscale(cadd(zk, zc), 0.5f);
        const float2 d = csub(zk, zc);
        const float2 odd = make_float2(0.5f * d.y, -0.5f * d.x);
        const float2 wk = c_tw[k << (TW_LOG - LOGN - 1)];
        colbuf[e] = cadd(even, cmul(wk, odd));
    }
    __syncthreads();

    // ---- columns: HW-point FFT of each decimated sequence X[Q a + b][c], a < HW
    for (int e = tid; e < w * Q; e += blockDim.x) {
        const int c = e % w, b = e / w;
        float2 v[HW];
#pragma unroll
        for (int a = 0; a < HW; a++) v[a] = colbuf[(size_t)(Q * a + b) * w + c];
        fftRegDIF<HW>(v);
        float2* dst = exch + ((size_t)c * Q + b) * HW;
#pragma unroll
        for (int i = 0; i < HW; i++) dst[brevC<LOGHW>(i)] = v[i];
    }
    __syncthreads();

    // ---- kept rows: Y[k] = sum_b exp(-2 pi i k b / H) Z_b[k mod HW], then the window operations
    float2 bc = make_float2(1.0f, 0.0f);
    if (p.batchCal && p.batchCalCount > 0)
        bc = p.batchCal[pol * p.batchCalCount + ((p.frameOffset + frame) % p.batchCalCount)];
    const float kx0 = p.kx0[pol], ky0 = p.ky0[pol], r02 = p.r02[pol];
    const float bcx = p.bcx[pol], bcy = p.bcy[pol];
    const int twShiftH = TW_LOG - p.logH;
    for (int e = tid; e < p.h * w; e += blockDim.x) {
        const int j = e / w, c = e - j * w;
        const int jSY = j + p.sy[pol];
        const int row = wrapModF(jSY + H / 2, H);
        const float2* zb = exch + (size_t)c * Q * HW + (row & (HW - 1));
        float2 Y = zb[0];
        for (int b = 1; b < Q; b++) {
            const float2 t = c_tw[((row * b) & (H - 1)) << twShiftH];
            Y = cadd(Y, cmul(zb[(size_t)b * HW], t));
        }
        Y = cmul(Y, bc);
        const float kx = p.kxAxis[sx0 + c];
        const float ky = p.kyAxis[row];
        const float shift = jSY < 0 ? p.kyShift : (jSY > H ? -p.kyShift : 0.0f);
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
        const size_t o = ((size_t)(frame * p.polCount + pol) * p.h + j) * p.w + c;
        p.window[o] = cmul(Y, adj);
    }
}

cudaError_t dh_forward_reg_init(const float2* hostTwiddle) {
    return cudaMemcpyToSymbol(c_tw, hostTwiddle, sizeof(float2) * TW_N);
}

template <int N, int HW>
static cudaError_t launchReg(const DhFwdParams& p, cudaStream_t s) {
    const int H = 1 << p.logH;
    const int threads = max(H, p.w * (H / HW));
    const size_t smem = sizeof(float2) * ((size_t)H * (N + 1) + (size_t)H * p.w);
    const size_t exch = sizeof(float2) * (size_t)p.w * (H / HW) * HW;
    if (exch > sizeof(float2) * (size_t)H * (N + 1)) return cudaErrorNotSupported;
    cudaError_t e = cudaFuncSetAttribute(k_forward_reg<N, HW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_forward_reg<N, HW><<<(unsigned)(p.frameCount * p.polCount), threads, smem, s>>>(p);
    return cudaGetLastError();
}

// Returns cudaErrorNotSupported when the shape needs the generic kernel.
cudaError_t dh_launch_forward_reg(const DhFwdParams& p, cudaStream_t s) {
    const int W = 1 << p.logW, H = 1 << p.logH;
    if (p.h != p.w || H > 256 || H < p.h || p.w > 32) return cudaErrorNotSupported;
    if (p.w * (H / p.h) > 256) return cudaErrorNotSupported;
    const size_t smem = sizeof(float2) * ((size_t)H * (W / 2 + 1) + (size_t)H * p.w);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    if (p.h == 16) {
        if (W == 32) return launchReg<16, 16>(p, s);
        if (W == 64) return launchReg<32, 16>(p, s);
        if (W == 128) return launchReg<64, 16>(p, s);
    } else if (p.h == 32) {
        if (W == 64) return launchReg<32, 32>(p, s);
        if (W == 128) return launchReg<64, 32>(p, s);
    }
    return cudaErrorNotSupported;
}
