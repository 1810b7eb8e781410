// Forward stage, register-resident variant for FFT windows up to 128 pixels
// wide (same results as k_forward in dh_kernels.cu, and as the reference's
// FFTW r2c + digHoloCopyWindow, digHolo.cpp:7184-7260 and 1808-2122).
//
//   1. the window is staged into shared memory with coalesced 16-byte loads;
//   2. two threads share a row: after the first decimation-in-frequency
//      stage of the packed half-length complex FFT, each transforms one half
//      (even or odd outputs) in registers, with literal twiddles;
//   3. the R2C split is evaluated for the IFFT window's kx columns only;
//   4. the column transform is evaluated for the IFFT window's h rows only:
//      h-point register FFTs of the H/h decimated column sequences, then an
//      H/h-term twiddled sum;
//   5. the frame-independent window factors (mask, normalisation, inverse
//      pixel sinc, beam-centre phase) come from a per-configuration table.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_params.h"
#include "dh_twiddle128.h"

using namespace dh;

namespace {

// In-place radix-2 decimation-in-frequency FFT of N <= 64 values in
// registers: natural-order input, bit-reversed output.
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
                if (j == 0) {
                    v[blk + j + m] = d;
                } else if (2 * j == m) {
                    v[blk + j + m] = make_float2(d.y, -d.x);  // multiply by -i
                } else {
                    v[blk + j + m] = cmul(d, tw64(j * (64 / (2 * m))));
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

// uint16 -> float without the conversion unit: 2^23 + u has the integer u in
// its mantissa, so subtracting 2^23 is exact.
__device__ __forceinline__ float u16lo(unsigned int u) { return __int_as_float(0x4B000000u | (u & 0xFFFFu)) - 8388608.0f; }
__device__ __forceinline__ float u16hi(unsigned int u) { return __int_as_float(0x4B000000u | (u >> 16)) - 8388608.0f; }

// Pixel pairs 4q .. 4q+3 (pixels 8q .. 8q+7 for uint16, 4q .. 4q+3 pairs for
// float) of a staged row, read with one or two 16-byte shared loads.
template <bool U16>
__device__ __forceinline__ void pixelQuad(const unsigned char* row, int q, float2 (&out)[4]) {
    if (U16) {
        const uint4 u = *reinterpret_cast<const uint4*>(row + 16 * q);
        out[0] = make_float2(u16lo(u.x), u16hi(u.x));
        out[1] = make_float2(u16lo(u.y), u16hi(u.y));
        out[2] = make_float2(u16lo(u.z), u16hi(u.z));
        out[3] = make_float2(u16lo(u.w), u16hi(u.w));
    } else {
        const float4 a = *reinterpret_cast<const float4*>(row + 32 * q);
        const float4 b = *reinterpret_cast<const float4*>(row + 32 * q + 16);
        out[0] = make_float2(a.x, a.y);
        out[1] = make_float2(a.z, a.w);
        out[2] = make_float2(b.x, b.y);
        out[3] = make_float2(b.z, b.w);
    }
}

}  // namespace

// N: complex samples per packed row (W/2).  HW: IFFT-window height h.
// blockDim.x = 2H; one block per (frame, polarisation).
template <int N, int HW, bool U16>
__global__ void __launch_bounds__(256, 2) k_forward_reg(DhFwdParams p) {
    constexpr int HALF = N / 2;
    constexpr int LOGHALF = ilog2c(HALF);
    constexpr int LOGHW = ilog2c(HW);
    constexpr int ZLD = N + 2;                  // Z row stride (complex), padded: conflict-free pair stores
    constexpr int ES = U16 ? 2 : 4;
    constexpr int ROWBYTES = 2 * N * ES;
    constexpr int SLD = ROWBYTES + 16;          // staging row stride (bytes), padded
    extern __shared__ float4 smRaw[];
    const int H = 1 << p.logH;
    const int w = p.w, h = p.h;
    const int Q = H / HW;
    const int unit = blockIdx.x;
    const int pol = unit % p.polCount;
    const int frame = unit / p.polCount;
    const int tid = threadIdx.x;

    unsigned char* region = reinterpret_cast<unsigned char*>(smRaw);
    const size_t regionBytes = max((size_t)H * SLD, (size_t)H * ZLD * sizeof(float2));
    float2* colbuf = reinterpret_cast<float2*>(region + regionBytes);   // H x w
    float2* tSplit = colbuf + (size_t)H * w;                            // w
    float2* tCol = tSplit + w;                                          // h x Q
    float2* tAdj = tCol + (size_t)h * Q;                                // h x w

    // per-configuration tables
    for (int e = tid; e < w; e += blockDim.x) tSplit[e] = p.tabSplit[pol * w + e];
    for (int e = tid; e < h * Q; e += blockDim.x) tCol[e] = p.tabCol[(size_t)pol * h * Q + e];
    for (int e = tid; e < h * w; e += blockDim.x) tAdj[e] = p.tabAdj[(size_t)pol * h * w + e];

    // 1. coalesced staging of the H x W window
    {
        const unsigned char* src = static_cast<const unsigned char*>(p.frames) +
            ((size_t)frame * p.frameStride + (size_t)p.cy[pol] * p.frameWidth + p.cx[pol]) * ES;
        const size_t srcPitch = (size_t)p.frameWidth * ES;
        constexpr int VPR = ROWBYTES / 16;
        for (int e = tid; e < H * VPR; e += blockDim.x) {
            const int r = e / VPR, q = e - r * VPR;
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + r * srcPitch) + q);
            *reinterpret_cast<uint4*>(region + (size_t)r * SLD + 16 * q) = v;
        }
    }
    __syncthreads();

    // 2. row transforms: thread pair (row r, half hf)
    const int r = tid >> 1, hf = tid & 1;
    float2 u[HALF];
    if (r < H) {
        const unsigned char* row = region + (size_t)r * SLD;
#pragma unroll
        for (int q = 0; q < HALF / 4; q++) {
            float2 a[4], b[4];
            pixelQuad<U16>(row, q, a);
            pixelQuad<U16>(row, q + HALF / 4, b);
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int j = 4 * q + t;
                u[j] = hf ? cmul(csub(a[t], b[t]), tw64(j * (64 / N))) : cadd(a[t], b[t]);
            }
        }
        fftRegDIF<HALF>(u);
    }
    __syncthreads();  // staging is dead; Z overwrites it
    float2* zbuf = reinterpret_cast<float2*>(region);
    if (r < H) {
        float2* zr = zbuf + (size_t)r * ZLD;
#pragma unroll
        for (int i = 0; i < HALF; i++) zr[2 * brevC<LOGHALF>(i) + hf] = u[i];
    }
    __syncthreads();

    // 3. R2C split for the kept columns k = sx0 + c
    const int sx0 = p.sx0[pol];
    for (int e = tid; e < H * w; e += blockDim.x) {
        const int rr = e / w, c = e - rr * w;
        const int k = sx0 + c;
        const float2* zr = zbuf + (size_t)rr * ZLD;
        const float2 zk = zr[k & (N - 1)];
        const float2 zc = cconj(zr[(N - k) & (N - 1)]);
        const float2 even = cscale(cadd(zk, zc), 0.5f);
        const float2 d = csub(zk, zc);
        const float2 odd = make_float2(0.5f * d.y, -0.5f * d.x);
        colbuf[e] = cadd(even, cmul(tSplit[c], odd));
    }
    __syncthreads();

    // 4. column transforms of the decimated sequences X[Q a + b][c], a < HW
    float2* exch = zbuf;  // [HW][Q][w], after the split Z is dead
    for (int e = tid; e < w * Q; e += blockDim.x) {
        const int c = e % w, b = e / w;
        float2 v[HW];
#pragma unroll
        for (int a = 0; a < HW; a++) v[a] = colbuf[(size_t)(Q * a + b) * w + c];
        fftRegDIF<HW>(v);
#pragma unroll
        for (int i = 0; i < HW; i++) exch[((size_t)brevC<LOGHW>(i) * Q + b) * w + c] = v[i];
    }
    __syncthreads();

    // 5. kept rows: Y = sum_b tCol[j][b] Z_b[row mod HW], then the window factors
    float2 bc = make_float2(1.0f, 0.0f);
    if (p.batchCal && p.batchCalCount > 0)
        bc = p.batchCal[pol * p.batchCalCount + ((p.frameOffset + frame) % p.batchCalCount)];
    const int sy = p.sy[pol];
    float2* out = p.window + (size_t)(frame * p.polCount + pol) * h * w;
    for (int e = tid; e < h * w; e += blockDim.x) {
        const int j = e / w, c = e - j * w;
        int row = (j + sy + H / 2) % H;
        if (row < 0) row += H;
        const float2* zb = exch + (size_t)(row & (HW - 1)) * Q * w + c;
        const float2* tc = tCol + (size_t)j * Q;
        float2 Y = zb[0];
        for (int b = 1; b < Q; b++) Y = cadd(Y, cmul(zb[(size_t)b * w], tc[b]));
        out[e] = cmul(cmul(Y, bc), tAdj[e]);
    }
}

template <int N, int HW>
static cudaError_t launchReg(const DhFwdParams& p, cudaStream_t s) {
    const int H = 1 << p.logH;
    const int es = p.inputU16 ? 2 : 4;
    const size_t region = max((size_t)H * (2 * N * es + 16), (size_t)H * (N + 2) * sizeof(float2));
    const size_t smem = region + sizeof(float2) * ((size_t)H * p.w + p.w + (size_t)p.h * (H / HW) + (size_t)p.h * p.w);
    if ((size_t)p.w * H * sizeof(float2) > region) return cudaErrorNotSupported;
    const unsigned blocks = (unsigned)(p.frameCount * p.polCount);
    cudaError_t e;
    if (p.inputU16) {
        e = cudaFuncSetAttribute(k_forward_reg<N, HW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_forward_reg<N, HW, true><<<blocks, 2 * H, smem, s>>>(p);
    } else {
        e = cudaFuncSetAttribute(k_forward_reg<N, HW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_forward_reg<N, HW, false><<<blocks, 2 * H, smem, s>>>(p);
    }
    return cudaGetLastError();
}

// Returns cudaErrorNotSupported when the shape needs the generic kernel.
cudaError_t dh_launch_forward_reg(const DhFwdParams& p, cudaStream_t s) {
    const int W = 1 << p.logW, H = 1 << p.logH;
    if (!p.tabSplit || !p.tabCol || !p.tabAdj) return cudaErrorNotSupported;
    if (p.h != p.w || H > 128 || H < p.h || p.w > 32) return cudaErrorNotSupported;
    if (p.w * (H / p.h) > 2 * H) return cudaErrorNotSupported;
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
