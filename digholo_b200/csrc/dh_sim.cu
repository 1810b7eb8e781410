// Frame simulator kernels (digHoloFrameSimulatorCreate, digHolo.cpp:15930-16760
// with the per-frame routine digHolo.cpp:15706-15877 and
// generateModeSeparable, digHolo.cpp:1610-1760): the camera intensity
// |R + sum_mn c_mn HG_m HG_n|^2 of every frame and polarisation, optionally
// filtered by the pixel fill-factor sinc in Fourier space, then quantised to
// the camera's levels against the batch maximum.
//
// The field of a polarisation region is accumulated in the reference's
// order and float rounding: the first mode's term plus the reference wave,
// then every later mode with a nonzero coefficient (and the last mode) in
// mode order; a term is (float)(int16 column mode x int16 row mode) times
// the float coefficient c xScale yScale, with no fused multiply-add, and
// the reference wave is the complex product of its column and row factors
// with the reference's fused real part.  The intensity is re^2 + im^2.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_sim.h"

using namespace dh;

namespace {

constexpr int SIM_T = 256;   // threads per field block
constexpr int SIM_RB = 8;    // rows per field block

// One block: SIM_RB rows of one (frame, polarisation) region.
__global__ void __launch_bounds__(SIM_T) k_sim_field(DhSimFieldArgs a) {
    extern __shared__ float4 simSm[];
    DhSimMode* modes = reinterpret_cast<DhSimMode*>(simSm);
    const int rowBlocks = (a.rows + SIM_RB - 1) / SIM_RB;
    const int unit = blockIdx.x / rowBlocks, r0 = (blockIdx.x % rowBlocks) * SIM_RB;
    const int pol = unit % a.polCount, frame = unit / a.polCount;
    const int beg = a.modeOffset[unit], cnt = a.modeOffset[unit + 1] - beg;
    for (int e = threadIdx.x; e < cnt; e += SIM_T) modes[e] = a.modes[beg + e];
    __syncthreads();
    const short* hc = a.hgCol + (size_t)pol * a.G * a.cols;   // [G][cols]
    const short* hr = a.hgRow + (size_t)pol * a.G * a.rows;   // [G][rows]
    const float2* rc = a.refCol + (size_t)pol * a.cols;
    const float2* rr = a.refRow + (size_t)pol * a.rows;
    float vmax = 0.f;
    const int rows = min(SIM_RB, a.rows - r0);
    for (int e = threadIdx.x; e < rows * a.cols; e += SIM_T) {
        const int r = r0 + e / a.cols, c = e % a.cols;
        float2 f = make_float2(0.f, 0.f);
        for (int k = 0; k < cnt; k++) {
            const DhSimMode md = modes[k];
            const int prod = (int)__ldg(&hc[(size_t)md.m * a.cols + c]) * (int)__ldg(&hr[(size_t)md.n * a.rows + r]);
            const float v = __int2float_rn(prod);
            const float2 t = make_float2(__fmul_rn(v, md.cr), __fmul_rn(v, md.ci));
            if (k == 0) {
                // generateModeSeparable: ref + V for the first mode (cmul's real part fused)
                const float2 x = rc[c], y = rr[r];
                const float2 ref = make_float2(fmaf(x.x, y.x, -__fmul_rn(x.y, y.y)), fmaf(x.x, y.y, __fmul_rn(x.y, y.x)));
                f = make_float2(__fadd_rn(ref.x, t.x), __fadd_rn(ref.y, t.y));
            } else {
                f = make_float2(__fadd_rn(t.x, f.x), __fadd_rn(t.y, f.y));
            }
        }
        const float I = __fadd_rn(__fmul_rn(f.x, f.x), __fmul_rn(f.y, f.y));
        a.out[(size_t)frame * a.rows * a.frameWidth + (size_t)r * a.frameWidth + (size_t)pol * a.cols + c] = I;
        vmax = fmaxf(vmax, I);
    }
    // non-negative floats order like their bit patterns
    for (int off = 16; off > 0; off >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
    if ((threadIdx.x & 31) == 0) atomicMax(a.maxBits, __float_as_uint(vmax));
}

// Basis fields (GetFieldsBasis, digHolo.cpp:5233-5305, through
// generateModeSeparable without the transpose or a reference wave): field
// [mode][pol][rows][cols] = sum over the mode's terms of (float)(int16 x
// mode x int16 y mode) c in the same order and rounding as k_sim_field.
__global__ void __launch_bounds__(SIM_T) k_basis_fields(DhSimFieldArgs a, float2* out) {
    extern __shared__ float4 bfSm[];
    DhSimMode* modes = reinterpret_cast<DhSimMode*>(bfSm);
    const int rowBlocks = (a.rows + SIM_RB - 1) / SIM_RB;
    const int unit = blockIdx.x / rowBlocks, r0 = (blockIdx.x % rowBlocks) * SIM_RB;
    const int pol = unit % a.polCount;
    const int beg = a.modeOffset[unit], cnt = a.modeOffset[unit + 1] - beg;
    for (int e = threadIdx.x; e < cnt; e += SIM_T) modes[e] = a.modes[beg + e];
    __syncthreads();
    const short* hc = a.hgCol + (size_t)pol * a.G * a.cols;
    const short* hr = a.hgRow + (size_t)pol * a.G * a.rows;
    const int rows = min(SIM_RB, a.rows - r0);
    for (int e = threadIdx.x; e < rows * a.cols; e += SIM_T) {
        const int r = r0 + e / a.cols, c = e % a.cols;
        float2 f = make_float2(0.f, 0.f);
        for (int k = 0; k < cnt; k++) {
            const DhSimMode md = modes[k];
            const int prod = (int)__ldg(&hc[(size_t)md.m * a.cols + c]) * (int)__ldg(&hr[(size_t)md.n * a.rows + r]);
            const float v = __int2float_rn(prod);
            const float2 t = make_float2(__fmul_rn(v, md.cr), __fmul_rn(v, md.ci));
            f = k == 0 ? t : make_float2(__fadd_rn(t.x, f.x), __fadd_rn(t.y, f.y));
        }
        out[((size_t)unit * a.rows + r) * a.cols + c] = f;
    }
}

// X[ky][kx] *= (sincY[ky] norm) sincX[kx] on [frame][H][W/2+1].
__global__ void k_sim_sinc(float2* X, int frames, int H, int Nx, const float* sincX, const float* sincY, float norm) {
    const size_t total = (size_t)frames * H * Nx;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int kx = (int)(e % Nx), ky = (int)((e / Nx) % H);
        const float env = __fmul_rn(__fmul_rn(sincY[ky], norm), sincX[kx]);
        X[e] = make_float2(__fmul_rn(X[e].x, env), __fmul_rn(X[e].y, env));
    }
}

// Rows of the half spectrum [frame][H][W/2+1] extended by Hermitian symmetry
// to [frame][H][W]: X[k] = conj(X[W - k]) for k > W/2.
__global__ void k_sim_extend(const float2* __restrict__ half, float2* full, int frames, int H, int W) {
    const int Nx = W / 2 + 1;
    const size_t total = (size_t)frames * H * W;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % W);
        const size_t row = e / W;
        full[e] = k < Nx ? half[row * Nx + k] : cconj(half[row * Nx + (W - k)]);
    }
}

__global__ void k_sim_real(const float2* __restrict__ full, float* out, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        out[e] = full[e].x;
}

// Quantisation against the batch maximum (digHolo.cpp:15847-15873):
// v = round-half-even(I (levels - 1) / max), kept as float and saturated to
// uint16.
__global__ void k_sim_quant(float* frames, unsigned short* frames16, size_t n, const unsigned* maxBits, int levels) {
    const float maxV = __uint_as_float(*maxBits);
    const float inv = __fdiv_rn((float)(levels - 1), maxV);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float v = rintf(__fmul_rn(frames[e], inv));
        frames[e] = v;
        if (frames16) frames16[e] = (unsigned short)min(max(__float2int_rn(v), 0), 65535);
    }
}

int gridFor(size_t n) {
    size_t g = (n + 255) / 256;
    return (int)(g > 148 * 32 ? 148 * 32 : (g < 1 ? 1 : g));
}

}  // namespace

cudaError_t dh_launch_sim_field(const DhSimFieldArgs& a, int maxModesPerUnit, cudaStream_t s) {
    const int units = a.frames * a.polCount;
    if (units <= 0) return cudaSuccess;
    const size_t smem = sizeof(DhSimMode) * (size_t)(maxModesPerUnit > 0 ? maxModesPerUnit : 1);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_sim_field), (int)smem);
    if (e != cudaSuccess) return e;
    const int rowBlocks = (a.rows + SIM_RB - 1) / SIM_RB;
    k_sim_field<<<(unsigned)(units * rowBlocks), SIM_T, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t dh_launch_basis_fields(const DhSimFieldArgs& a, int maxModesPerUnit, float2* out, cudaStream_t s) {
    const int units = a.frames * a.polCount;
    if (units <= 0) return cudaSuccess;
    const size_t smem = sizeof(DhSimMode) * (size_t)(maxModesPerUnit > 0 ? maxModesPerUnit : 1);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_basis_fields), (int)smem);
    if (e != cudaSuccess) return e;
    const int rowBlocks = (a.rows + SIM_RB - 1) / SIM_RB;
    k_basis_fields<<<(unsigned)(units * rowBlocks), SIM_T, smem, s>>>(a, out);
    return cudaGetLastError();
}

cudaError_t dh_launch_sim_sinc(float2* X, int frames, int H, int Nx, const float* sincX, const float* sincY, float norm,
                               cudaStream_t s) {
    k_sim_sinc<<<gridFor((size_t)frames * H * Nx), 256, 0, s>>>(X, frames, H, Nx, sincX, sincY, norm);
    return cudaGetLastError();
}

cudaError_t dh_launch_sim_extend(const float2* half, float2* full, int frames, int H, int W, cudaStream_t s) {
    k_sim_extend<<<gridFor((size_t)frames * H * W), 256, 0, s>>>(half, full, frames, H, W);
    return cudaGetLastError();
}

cudaError_t dh_launch_sim_real(const float2* full, float* out, size_t n, cudaStream_t s) {
    k_sim_real<<<gridFor(n), 256, 0, s>>>(full, out, n);
    return cudaGetLastError();
}

cudaError_t dh_launch_sim_quant(float* frames, unsigned short* frames16, size_t n, const unsigned* maxBits, int levels,
                                cudaStream_t s) {
    k_sim_quant<<<gridFor(n), 256, 0, s>>>(frames, frames16, n, maxBits, levels);
    return cudaGetLastError();
}
