// Pieces shared by the full-resolution field kernels: register-resident
// radix-2 inverse FFTs, the field-statistics record and its merge rule, and
// the positive-exponent twiddle lookup.
#pragma once
#include <cuda_runtime.h>

#include "dh_common.cuh"
#include "dh_twiddle128.h"

namespace dh {
template <int LOG>
__host__ __device__ constexpr int brevF(int i) {
    int r = 0;
    for (int b = 0; b < LOG; b++) r |= ((i >> b) & 1) << (LOG - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2F(int n) { return n <= 1 ? 0 : 1 + ilog2F(n / 2); }

// In-place radix-2 DIF inverse FFT (exp(+2 pi i / N), unnormalised), N <= 64:
// natural-order input, bit-reversed output.
template <int N>
__device__ __forceinline__ void ifftDIFf(float2 (&v)[N]) {
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
                    v[blk + j + m] = make_float2(-d.y, d.x);
                } else {
                    const float2 t = tw128(j * (128 / (2 * m)));
                    v[blk + j + m] = cmul(d, make_float2(t.x, -t.y));
                }
            }
        }
    }
}

struct StatF {
    float maxI;
    int maxIdx;
    float P, cx, cy, cyw, e4;
};

__device__ __forceinline__ void statMerge(StatF& a, float mI, int mIdx, float P, float cx, float cy, float cyw, float e4) {
    if (mI > a.maxI || (mI == a.maxI && mIdx > a.maxIdx)) { a.maxI = mI; a.maxIdx = mIdx; }
    a.P += P; a.cx += cx; a.cy += cy; a.cyw += cyw; a.e4 += e4;
}

// e^{+2 pi i n / N} from the table exp(-2 pi i k / 4096)
__device__ __forceinline__ float2 expPos(const float2* __restrict__ tw, int n, int N) {
    const float2 t = __ldg(&tw[(n & (N - 1)) * (TW_N / N)]);
    return make_float2(t.x, -t.y);
}


}  // namespace dh
