// Shared device helpers for the digholo_b200 kernels: complex arithmetic,
// the twiddle table and an in-place radix-2 FFT over batches of sequences
// held in shared memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dh {

// Length of the global twiddle table: twiddle(k) = exp(-2 pi i k / TW_N).
// Every power-of-two transform length N <= TW_N reads it with stride TW_N / N.
constexpr int TW_N = 4096;
constexpr int TW_LOG = 12;

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

__device__ __forceinline__ int bitrev(int i, int logn) {
    return logn == 0 ? 0 : (int)(__brev((unsigned)i) >> (32 - logn));
}

// In-place radix-2 decimation-in-time FFT of `count` sequences of length
// 2^logn in shared memory.  Element i of sequence s lives at
// base[s * seqStride + i * elemStride]; the input must be in bit-reversed
// order and the output is in natural order.  inverse = false uses
// exp(-2 pi i / N) (FFTW_FORWARD), inverse = true exp(+2 pi i / N)
// (FFTW_BACKWARD); both are unnormalised.  When `colMajor` is set,
// consecutive threads take consecutive sequences (use it when seqStride is 1
// so that a warp touches consecutive words).  All threads of the block must
// call this; it ends with a barrier.
__device__ __forceinline__ void fft_dit(float2* base, int count, int seqStride, int elemStride,
                                        int logn, bool inverse, bool colMajor,
                                        const float2* __restrict__ tw) {
    const int n = 1 << logn;
    const int halfN = n >> 1;
    const int total = count * halfN;
    for (int lh = 0; lh < logn; lh++) {
        const int half = 1 << lh;
        // twiddle exp(-2 pi i j / (2 half)) = tw[j << (TW_LOG - lh - 1)]
        const int twShift = TW_LOG - lh - 1;
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            int s, b;
            if (colMajor) { s = t % count; b = t / count; }
            else { s = t >> (logn - 1); b = t & (halfN - 1); }
            const int j = b & (half - 1);
            const int i0 = ((b >> lh) << (lh + 1)) + j;
            const int i1 = i0 + half;
            float2 w = __ldg(&tw[j << twShift]);
            if (inverse) w.y = -w.y;
            float2* p = base + (size_t)s * seqStride;
            const float2 a = p[i0 * elemStride];
            const float2 c = cmul(p[i1 * elemStride], w);
            p[i0 * elemStride] = cadd(a, c);
            p[i1 * elemStride] = csub(a, c);
        }
        __syncthreads();
    }
}

// Round half to even and saturate to int16, as the reference's
// _mm256_cvtps_epi32 + _mm256_packs_epi32 do (digHolo.cpp:2822-2829): NaN
// gives INT_MIN there and so -32768 here (fmaxf returns the non-NaN operand).
// Inputs are scale * v with |scale * v| <= 32767 (1 + 2^-13) for finite
// fields, so the int32 overflow cases of the conversion never arise.  The
// clamped value plus 1.5 * 2^23 carries the rounded integer in its low bits.
__device__ __forceinline__ short roundSat16(float v) {
    const float c = fminf(fmaxf(v, -32768.0f), 32767.0f);
    return (short)__float_as_int(c + 12582912.0f);
}

// x / sin(x) with value 1 at x = 0: the inverse pixel sinc used for the
// fill-factor correction.
__device__ __forceinline__ float xcsc(float x) {
    return x == 0.0f ? 1.0f : x / sinf(x);
}

}  // namespace dh
