// Reference-wave calibration planes (digHolo.cpp:6729-6830, 8253-8285): the
// stored calibration frames go through a c2c FFT of the frames' FFT windows,
// the Fourier window at zero tilt, and an IFFT of the field's size.  This
// runs once per calibration and geometry, so the transforms are plain
// separable DFTs evaluated only where they are needed (the window's kx
// columns and ky rows going forward, the field's pixels going back), each
// output an FP64 sum over one axis rounded to FP32, like the FP32 FFTs of
// the reference to within their rounding.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_params.h"

namespace {

constexpr int CAL_THREADS = 256;

// Reference's complex product, real part fused (digHolo.cpp:885-892).
__device__ __forceinline__ float2 cmulFused(float2 a, float2 b) {
    return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}

__global__ void __launch_bounds__(CAL_THREADS) k_cal_dft(DhCalDft q) {
    extern __shared__ double2 tw[];   // exp(sign 2 pi i r / N), r < N
    for (int r = threadIdx.x; r < q.N; r += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)r / (double)q.N, &s, &c);
        tw[r] = make_double2(c, q.sign > 0 ? s : -s);
    }
    __syncthreads();
    const long long total = (long long)q.U * q.A * q.B;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e % q.B);
        const long long ua = e / q.B;
        const int a = (int)(ua % q.A);
        const int u = (int)(ua / q.A);
        const int pu = u % q.fP;
        const int oi = q.outOnA ? a : b;
        const long long fo = q.freqOut ? q.freqOut[(size_t)pu * (q.outOnA ? q.A : q.B) + oi] : oi;
        const int* fk = q.freqK ? q.freqK + (size_t)pu * q.K : nullptr;
        const float2* src = q.in + u * q.inU + a * q.inA + b * q.inB;
        double ar = 0.0, ai = 0.0;
        for (int k = 0; k < q.K; k++) {
            const float2 v = src[k * q.inK];
            const long long f = fk ? fk[k] : k;
            const double2 t = tw[(int)((fo * f) % q.N)];
            ar = fma((double)v.x, t.x, fma(-(double)v.y, t.y, ar));
            ai = fma((double)v.x, t.y, fma((double)v.y, t.x, ai));
        }
        float2 r = make_float2((float)ar, (float)ai);
        if (q.ufac) r = cmulFused(r, q.ufac[u]);
        if (q.fac) {
            const float f = q.fac[((size_t)pu * q.A + a) * q.B + b];
            r = make_float2(__fmul_rn(r.x, f), __fmul_rn(r.y, f));
        }
        q.out[e] = r;
    }
}

}  // namespace

cudaError_t dh_launch_cal_dft(const DhCalDft& q, cudaStream_t s) {
    if (q.N <= 0 || q.N > 4096 || q.fP < 1 || q.U <= 0 || q.A <= 0 || q.B <= 0 || q.K <= 0)
        return cudaErrorInvalidValue;
    const size_t smem = sizeof(double2) * (size_t)q.N;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_cal_dft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const long long total = (long long)q.U * q.A * q.B;
    long long blocks = (total + CAL_THREADS - 1) / CAL_THREADS;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_cal_dft<<<(unsigned)blocks, CAL_THREADS, smem, s>>>(q);
    return cudaGetLastError();
}
