// Adjoint of the batch path for gradient-driven AutoAlign: the gradient of
// the captured power S = sum |c_mn|^2 (IL = 10 log10 S + const, the power
// meter's insertion loss, digHolo.cpp:3105-3143 and 11012-11062) with
// respect to each polarisation's beam centre, tilt, defocus and basis waist,
// with the Fourier-window selection held fixed.
//
// With V = -conj(A R) the tilt-removed field (A the reconstructed field, R
// the reference wave of digHolo.cpp:10386-10504, phase
//   phi(x, y) = (-k0 tx + offx) x + bcx (-k0 tx) + focal x^2 + (same in y),
//   focal = -pi D / lambda),
// and c_mn = sum_xy Hx_m(x) Hy_n(y) V(x, y) (the separable overlap,
// digHolo.cpp:2149-2341, in float), dS = 2 Re sum_mn conj(c_mn) dc_mn
//   = 2 Re sum_xy Abar dV + 2 Re sum_xy Abar_w dw V,
// Abar = sum_mn conj(c_mn) Hx_m Hy_n (the adjoint field) and
// Abar_w = sum_mn conj(c_mn) d(Hx_m Hy_n)/dw.  The tangents of V are
//   dV/dtx = V i k0 u (x + bcx),   dV/dty = V i k0 u (y + bcy)   (u = pi/180),
//   dV/dD  = V i (pi / lambda) (x^2 + y^2),
//   dV/dbcx = -conj(A_x R) + V i k0 u tx,  A_x the field of the window times
//             i kx (the beam-centre phase of digHoloCopyWindow, digHolo.cpp:1955-2035),
// and for the waist the Hermite-Gaussian ladder relation
//   dpsi_m/dw = -(1 / 2w) (sqrt(m (m-1)) psi_{m-2} - sqrt((m+1)(m+2)) psi_{m+2}).
// One block per (frame, polarisation) field; per-field partial sums of
// Re sum conj(c) dc for the six parameters and the field's sum |c|^2.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_grad.h"
#include "dh_host.h"

using namespace dh;


// Window of the beam-centre derivatives: Wx = i kx W, Wy = i ky W.
__global__ void k_window_deriv(const float2* __restrict__ W, const float* __restrict__ kxw, const float* __restrict__ kyw,
                               int w, int h, int polCount, int units, float2* __restrict__ Wx, float2* __restrict__ Wy) {
    const size_t total = (size_t)units * w * h;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t unit = e / ((size_t)w * h);
        const int rem = (int)(e - unit * w * h);
        const int j = rem / w, c = rem - j * w;
        const int pol = (int)(unit % polCount);
        const float2 v = W[e];
        const float kx = kxw[pol * w + c], ky = kyw[pol * h + j];
        Wx[e] = make_float2(-kx * v.y, kx * v.x);
        Wy[e] = make_float2(-ky * v.y, ky * v.x);
    }
}

// blockDim.x = 256; shared: U, Uw [G][ny] complex, hx/hy derivative rows.
__global__ void __launch_bounds__(256) k_align_grad(DhGradParams p) {
    extern __shared__ float2 sg[];
    const int unit = blockIdx.x;
    const int P = p.polCount, G = p.G, M = p.M, nx = p.nx, ny = p.ny;
    const int pol = unit % P, frame = unit / P;
    const int GE = G + 2;
    float2* cc = sg;                                   // [M] conj(c)
    float2* U = cc + M;                                // [G][ny]  sum_n conj(c_mn) Hy_n(y)
    float2* Uw = U + (size_t)G * ny;                   // [G][ny]  sum_n conj(c_mn) Hy'_n(y)
    float* dhx = reinterpret_cast<float*>(Uw + (size_t)G * ny);   // [G][nx] Hx'_m
    float* dhy = dhx + (size_t)G * nx;                              // [G][ny] Hy'_n
    float* red = dhy + (size_t)G * ny;                              // [8 warps][7]
    const float* hxp = p.hx + (size_t)pol * GE * nx;
    const float* hyp = p.hy + (size_t)pol * GE * ny;
    const float w0 = p.waist[pol];
    const int tid = threadIdx.x;

    float spow = 0.f;   // captured power of this field
    for (int mode = tid; mode < M; mode += blockDim.x) {
        const size_t ci = (size_t)frame * P * M + (size_t)pol * M + mode;
        const float2 c = p.coefs[ci];
        cc[mode] = p.weights ? p.weights[ci] : make_float2(c.x, -c.y);
        spow = fmaf(c.x, c.x, fmaf(c.y, c.y, spow));
    }
    // ladder derivatives of the modes with respect to the waist
    for (int e = tid; e < G * nx; e += blockDim.x) {
        const int m = e / nx, x = e - m * nx;
        float v = 0.f;
        if (m >= 2) v += sqrtf((float)(m * (m - 1))) * hxp[(m - 2) * nx + x];
        v -= sqrtf((float)((m + 1) * (m + 2))) * hxp[(m + 2) * nx + x];
        dhx[e] = -v / (2.0f * w0);
    }
    for (int e = tid; e < G * ny; e += blockDim.x) {
        const int n = e / ny, y = e - n * ny;
        float v = 0.f;
        if (n >= 2) v += sqrtf((float)(n * (n - 1))) * hyp[(n - 2) * ny + y];
        v -= sqrtf((float)((n + 1) * (n + 2))) * hyp[(n + 2) * ny + y];
        dhy[e] = -v / (2.0f * w0);
    }
    __syncthreads();
    // U[m][y] = sum_n conj(c_mn) Hy_n(y) over the modes m + n < G (digHolo.cpp:1245-1265 order)
    for (int e = tid; e < G * ny; e += blockDim.x) {
        const int m = e / ny, y = e - m * ny;
        float2 u = make_float2(0.f, 0.f), uw = make_float2(0.f, 0.f);
        for (int n = 0; m + n < G; n++) {
            const int g = m + n;
            const float2 c = cc[g * (g + 1) / 2 + n];
            const float hv = hyp[n * ny + y], dv = dhy[n * ny + y];
            u.x = fmaf(c.x, hv, u.x); u.y = fmaf(c.y, hv, u.y);
            uw.x = fmaf(c.x, dv, uw.x); uw.y = fmaf(c.y, dv, uw.y);
        }
        U[e] = u;
        Uw[e] = uw;
    }
    __syncthreads();

    const float2* Vp = p.V + (size_t)unit * nx * ny;
    const float2* Vxp = p.Vx + (size_t)unit * nx * ny;
    const float2* Vyp = p.Vy + (size_t)unit * nx * ny;
    const float k0u = p.k0u[pol];
    const float txr = p.tiltX[pol], tyr = p.tiltY[pol];
    const float bx = p.bcx[pol], by = p.bcy[pol];
    float s[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, spow};
    for (int e = tid; e < nx * ny; e += blockDim.x) {
        const int y = e / nx, x = e - y * nx;
        float2 a = make_float2(0.f, 0.f), aw = make_float2(0.f, 0.f);
        for (int m = 0; m < G; m++) {
            const float hv = hxp[m * nx + x], dv = dhx[m * nx + x];
            const float2 u = U[m * ny + y], uw = Uw[m * ny + y];
            a.x = fmaf(hv, u.x, a.x); a.y = fmaf(hv, u.y, a.y);
            aw.x = fmaf(dv, u.x, fmaf(hv, uw.x, aw.x));
            aw.y = fmaf(dv, u.y, fmaf(hv, uw.y, aw.y));
        }
        const float2 v = Vp[e], vx = Vxp[e], vy = Vyp[e];
        // Re(Abar V i) = -Im(Abar V)
        const float imAV = a.x * v.y + a.y * v.x;
        const float xv = p.xAxis[x], yv = p.yAxis[y];
        s[0] += -imAV * k0u * (xv + bx);
        s[1] += -imAV * k0u * (yv + by);
        s[2] += -imAV * p.piOverLambda * (xv * xv + yv * yv);
        s[3] += (a.x * vx.x - a.y * vx.y) - imAV * k0u * txr;
        s[4] += (a.x * vy.x - a.y * vy.y) - imAV * k0u * tyr;
        s[5] += aw.x * v.x - aw.y * v.y;
    }
#pragma unroll
    for (int k = 0; k < 7; k++)
        for (int off = 16; off > 0; off >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], off);
    if ((tid & 31) == 0)
        for (int k = 0; k < 7; k++) red[(tid >> 5) * 7 + k] = s[k];
    __syncthreads();
    if (tid < 7) {
        float t = 0.f;
        for (int wv = 0; wv < (int)(blockDim.x >> 5); wv++) t += red[wv * 7 + tid];
        p.out[(size_t)unit * 7 + tid] = t;
    }
}

// The same contraction for G <= GM, register-tiled: each thread owns one
// column x of the field, with Hx_m(x) and dHx_m/dw(x) for m < GM in
// registers, and walks the rows y = ty, ty + YS, ...; the row sums U[m][y]
// and Uw[m][y] sit in shared memory as one float4 per (m, y), which a warp
// (32 columns of one row) reads as a broadcast.  Rows G <= m < GM of the
// table are zero, so the unrolled mode loop needs no bound check.  Per pixel
// and mode: one shared load and six FMAs (the generic kernel above reads
// four values per pixel and mode).
template <int GM>
__global__ void __launch_bounds__(256) k_align_grad_reg(DhGradParams p) {
    extern __shared__ float4 sg4[];
    const int unit = blockIdx.x;
    const int P = p.polCount, G = p.G, M = p.M, nx = p.nx, ny = p.ny;
    const int pol = unit % P, frame = unit / P;
    const int GE = G + 2;
    float4* UU = sg4;                                                 // [GM][ny] {U, Uw}
    float2* cc = reinterpret_cast<float2*>(UU + (size_t)GM * ny);     // [M] conj(c)
    float* dhy = reinterpret_cast<float*>(cc + M);                    // [G][ny] Hy'_n
    float* red = dhy + (size_t)G * ny;                                // [8 warps][7]
    const float* hxp = p.hx + (size_t)pol * GE * nx;
    const float* hyp = p.hy + (size_t)pol * GE * ny;
    const float w0 = p.waist[pol];
    const float ladder = -1.0f / (2.0f * w0);
    const int tid = threadIdx.x;

    float spow = 0.f;
    for (int mode = tid; mode < M; mode += blockDim.x) {
        const size_t ci = (size_t)frame * P * M + (size_t)pol * M + mode;
        const float2 c = p.coefs[ci];
        cc[mode] = p.weights ? p.weights[ci] : make_float2(c.x, -c.y);
        spow = fmaf(c.x, c.x, fmaf(c.y, c.y, spow));
    }
    for (int e = tid; e < G * ny; e += blockDim.x) {
        const int n = e / ny, y = e - n * ny;
        float v = 0.f;
        if (n >= 2) v += sqrtf((float)(n * (n - 1))) * hyp[(n - 2) * ny + y];
        v -= sqrtf((float)((n + 1) * (n + 2))) * hyp[(n + 2) * ny + y];
        dhy[e] = v * ladder;
    }
    __syncthreads();
    for (int e = tid; e < GM * ny; e += blockDim.x) {
        const int m = e / ny, y = e - m * ny;
        float4 u = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int n = 0; m + n < G; n++) {
            const int g = m + n;
            const float2 c = cc[g * (g + 1) / 2 + n];
            const float hv = hyp[n * ny + y], dv = dhy[n * ny + y];
            u.x = fmaf(c.x, hv, u.x); u.y = fmaf(c.y, hv, u.y);
            u.z = fmaf(c.x, dv, u.z); u.w = fmaf(c.y, dv, u.w);
        }
        UU[e] = u;
    }
    __syncthreads();

    const size_t base = (size_t)unit * nx * ny;
    const float2* Vp = p.V + base;
    const float2* Vxp = p.Vx + base;
    const float2* Vyp = p.Vy + base;
    const int XT = nx < 256 ? nx : 256;   // nx is a power of two
    const int YS = 256 / XT;
    const int tx = tid % XT, ty = tid / XT;
    const float bx = p.bcx[pol], by = p.bcy[pol];
    // sums: Im(Abar V) (x + bcx), Im(Abar V) (y + bcy), Im(Abar V) (x^2 + y^2),
    // Re(Abar Vx), Re(Abar Vy), Re(Abar_w V), Im(Abar V)
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s4 = 0.f, s5 = 0.f, si = 0.f;
    for (int x0 = 0; x0 < nx; x0 += XT) {
        const int x = x0 + tx;
        float hr[GM], dr[GM];
#pragma unroll
        for (int m = 0; m < GM; m++) {
            hr[m] = 0.f;
            dr[m] = 0.f;
            if (m < G) {
                hr[m] = hxp[m * nx + x];
                float v = 0.f;
                if (m >= 2) v += sqrtf((float)(m * (m - 1))) * hxp[(m - 2) * nx + x];
                v -= sqrtf((float)((m + 1) * (m + 2))) * hxp[(m + 2) * nx + x];
                dr[m] = v * ladder;
            }
        }
        const float xv = p.xAxis[x];
        for (int y = ty; y < ny; y += YS) {
            const size_t e = (size_t)y * nx + x;
            const float2 v = Vp[e], vx = Vxp[e], vy = Vyp[e];
            float2 a = make_float2(0.f, 0.f), aw = make_float2(0.f, 0.f);
            const float4* Uy = UU + y;
#pragma unroll
            for (int m = 0; m < GM; m++) {
                const float4 u = Uy[m * ny];
                a.x = fmaf(hr[m], u.x, a.x);
                a.y = fmaf(hr[m], u.y, a.y);
                aw.x = fmaf(dr[m], u.x, fmaf(hr[m], u.z, aw.x));
                aw.y = fmaf(dr[m], u.y, fmaf(hr[m], u.w, aw.y));
            }
            const float imAV = a.x * v.y + a.y * v.x;
            const float yv = p.yAxis[y];
            s0 = fmaf(imAV, xv + bx, s0);
            s1 = fmaf(imAV, yv + by, s1);
            s2 = fmaf(imAV, xv * xv + yv * yv, s2);
            s3 += a.x * vx.x - a.y * vx.y;
            s4 += a.x * vy.x - a.y * vy.y;
            s5 += aw.x * v.x - aw.y * v.y;
            si += imAV;
        }
    }
    const float k0u = p.k0u[pol];
    // Re(Abar V i) = -Im(Abar V); the beam-centre tangents carry -Im(Abar V) k0 u t
    float s[7] = {-k0u * s0, -k0u * s1, -p.piOverLambda * s2, s3 - k0u * p.tiltX[pol] * si,
                  s4 - k0u * p.tiltY[pol] * si, s5, spow};
#pragma unroll
    for (int k = 0; k < 7; k++)
        for (int off = 16; off > 0; off >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], off);
    if ((tid & 31) == 0)
        for (int k = 0; k < 7; k++) red[(tid >> 5) * 7 + k] = s[k];
    __syncthreads();
    if (tid < 7) {
        float t = 0.f;
        for (int wv = 0; wv < (int)(blockDim.x >> 5); wv++) t += red[wv * 7 + tid];
        p.out[(size_t)unit * 7 + tid] = t;
    }
}

// The power term of the gradient kernels alone (their first loop and their
// block reduction, in the same order).
__global__ void __launch_bounds__(256) k_align_power(DhGradParams p) {
    __shared__ float red[8 * 7];
    const int unit = blockIdx.x;
    const int P = p.polCount, M = p.M;
    const int pol = unit % P, frame = unit / P;
    const int tid = threadIdx.x;
    float spow = 0.f;
    for (int mode = tid; mode < M; mode += blockDim.x) {
        const float2 c = p.coefs[(size_t)frame * P * M + (size_t)pol * M + mode];
        spow = fmaf(c.x, c.x, fmaf(c.y, c.y, spow));
    }
    float s[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, spow};
#pragma unroll
    for (int k = 0; k < 7; k++)
        for (int off = 16; off > 0; off >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], off);
    if ((tid & 31) == 0)
        for (int k = 0; k < 7; k++) red[(tid >> 5) * 7 + k] = s[k];
    __syncthreads();
    if (tid < 7) {
        float t = 0.f;
        for (int wv = 0; wv < (int)(blockDim.x >> 5); wv++) t += red[wv * 7 + tid];
        p.out[(size_t)unit * 7 + tid] = t;
    }
}

cudaError_t dh_launch_align_power(const DhGradParams& p, cudaStream_t s) {
    k_align_power<<<(unsigned)(p.frameCount * p.polCount), 256, 0, s>>>(p);
    return cudaGetLastError();
}

// Weights of an eigenvalue's derivative.  For an eigenpair (lambda, u) of
// the Gram matrix of the block A (rows = modes of pol0 [and pol1], columns
// = frames; column-major A[b rows + j]), d lambda = 2 Re sum_jb w_jb dA_jb
// with w_jb = conj(p_j) q_b and (p, q) = (u, A^H u) for the mode-space Gram
// A A^H, (A u, u) for the frame-space Gram A^H A.  W[b][pol M + m] +=
// alpha w_jb, row j < M of pol0, j >= M of pol1.  One thread per (j, b).
__global__ void k_mdl_weights(const float2* __restrict__ A, int rows, int batch, int rowsGram,
                              const double2* __restrict__ u, double alpha, int pol0, int pol1, int polCount, int M,
                              float2* __restrict__ W) {
    const int total = rows * batch;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int b = e / rows, j = e - b * rows;
        double2 pj, qb;
        if (rowsGram) {
            pj = u[j];
            double re = 0.0, im = 0.0;   // (A^H u)_b = sum_i conj(A_ib) u_i
            for (int i = 0; i < rows; i++) {
                const float2 a = A[(size_t)b * rows + i];
                re += (double)a.x * u[i].x + (double)a.y * u[i].y;
                im += (double)a.x * u[i].y - (double)a.y * u[i].x;
            }
            qb = make_double2(re, im);
        } else {
            double re = 0.0, im = 0.0;   // (A u)_j = sum_c A_jc u_c
            for (int c = 0; c < batch; c++) {
                const float2 a = A[(size_t)c * rows + j];
                re += (double)a.x * u[c].x - (double)a.y * u[c].y;
                im += (double)a.x * u[c].y + (double)a.y * u[c].x;
            }
            pj = make_double2(re, im);
            qb = u[b];
        }
        // conj(p_j) q_b
        const double wr = pj.x * qb.x + pj.y * qb.y, wi = pj.x * qb.y - pj.y * qb.x;
        const int pol = j < M ? pol0 : pol1, m = j < M ? j : j - M;
        float2* wp = W + (size_t)b * polCount * M + (size_t)pol * M + m;
        wp->x += (float)(alpha * wr);
        wp->y += (float)(alpha * wi);
    }
}

cudaError_t dh_launch_mdl_weights(const float2* A, int rows, int batch, int rowsGram, const double2* u, double alpha,
                                  int pol0, int pol1, int polCount, int M, float2* W, cudaStream_t s) {
    const int total = rows * batch;
    int blocks = (total + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    k_mdl_weights<<<blocks, 256, 0, s>>>(A, rows, batch, rowsGram, u, alpha, pol0, pol1, polCount, M, W);
    return cudaGetLastError();
}

cudaError_t dh_launch_window_deriv(const float2* W, const float* kxw, const float* kyw, int w, int h, int polCount, int units,
                                   float2* Wx, float2* Wy, cudaStream_t s) {
    const size_t total = (size_t)units * w * h;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    k_window_deriv<<<blocks, 256, 0, s>>>(W, kxw, kyw, w, h, polCount, units, Wx, Wy);
    return cudaGetLastError();
}

template <int GM>
static cudaError_t launchAlignGradReg(const DhGradParams& p, size_t smem, cudaStream_t s) {
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_align_grad_reg<GM>), (int)smem);
    if (e != cudaSuccess) return e;
    k_align_grad_reg<GM><<<(unsigned)(p.frameCount * p.polCount), 256, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t dh_launch_align_grad(const DhGradParams& p, cudaStream_t s) {
    const bool pow2 = p.nx > 0 && (p.nx & (p.nx - 1)) == 0;
    if (pow2 && p.G <= 32) {
        const int GM = p.G <= 16 ? 16 : 32;
        const size_t smemReg = sizeof(float4) * (size_t)GM * p.ny + sizeof(float2) * (size_t)p.M +
                               sizeof(float) * ((size_t)p.G * p.ny + 8 * 7);
        if (smemReg <= 200 * 1024) return GM == 16 ? launchAlignGradReg<16>(p, smemReg, s) : launchAlignGradReg<32>(p, smemReg, s);
    }
    const size_t smem = sizeof(float2) * ((size_t)p.M + 2 * (size_t)p.G * p.ny) + sizeof(float) * ((size_t)p.G * (p.nx + p.ny) + 8 * 7);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_align_grad), (int)smem);
    if (e != cudaSuccess) return e;
    k_align_grad<<<(unsigned)(p.frameCount * p.polCount), 256, smem, s>>>(p);
    return cudaGetLastError();
}
