// Power-meter support on the GPU: gather of one coefficient matrix block and
// its FP64 Gram matrix, whose eigenvalues (dh_eigen.cu, FP64) are the squared
// singular values digHolo takes from cgesvd (digHolo.cpp:3021-3055, used by
// digHoloPowerMeter digHolo.cpp:10980-11011).
#include <cuda_runtime.h>
#include <cuComplex.h>

#include <cstdio>

// Dense column-major block A (rows = svdM modes, cols = batch) from the
// coefficient array coefs[batch][polCount * M]:
//   row j < M      : src0[b][pol0 * M + j]
//   row j >= M     : src1[b][pol1 * M + (j - M)]   (only when rows == 2M)
__global__ void k_gather_block(const float2* __restrict__ src0, const float2* __restrict__ src1, int pol0, int pol1,
                               int polCount, int M, int rows, int batch, float2* __restrict__ A) {
    const int total = rows * batch;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int b = e / rows, j = e - b * rows;
        const float2* s = j < M ? src0 + (size_t)b * polCount * M + pol0 * M + j
                                : src1 + (size_t)b * polCount * M + pol1 * M + (j - M);
        A[(size_t)b * rows + j] = *s;
    }
}

// Gram matrix in FP64, column-major n x n:
//   rowsGram (n == rows):  G[i][k] = sum_b A[i][b] conj(A[k][b])
//   batch Gram (n == batch): G[i][k] = sum_j conj(A[j][i]) A[j][k]   (A^H A)
// One thread per (i, k) with 16 x 16 shared tiles of A.
__global__ void k_gram(const float2* __restrict__ A, int rows, int batch, int rowsGram, cuDoubleComplex* __restrict__ G) {
    __shared__ float2 ta[16][17];
    __shared__ float2 tb[16][17];
    const int n = rowsGram ? rows : batch;
    const int K = rowsGram ? batch : rows;
    const int i = blockIdx.y * 16 + threadIdx.y;
    const int k = blockIdx.x * 16 + threadIdx.x;
    double re = 0.0, im = 0.0;
    for (int t0 = 0; t0 < K; t0 += 16) {
        // ta[y][x] = element (i0 + y, t0 + x), tb[y][x] = element (k0 + y, t0 + x)
        const int ty = threadIdx.y, tx = threadIdx.x;
        const int ii = blockIdx.y * 16 + ty, kk = blockIdx.x * 16 + ty, tt = t0 + tx;
        float2 va = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
        if (tt < K) {
            if (rowsGram) {
                if (ii < n) va = A[(size_t)tt * rows + ii];
                if (kk < n) vb = A[(size_t)tt * rows + kk];
            } else {
                if (ii < n) va = A[(size_t)ii * rows + tt];
                if (kk < n) vb = A[(size_t)kk * rows + tt];
            }
        }
        ta[ty][tx] = va;
        tb[ty][tx] = vb;
        __syncthreads();
#pragma unroll
        for (int t = 0; t < 16; t++) {
            const float2 a = ta[threadIdx.y][t];
            const float2 b = tb[threadIdx.x][t];
            const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
            if (rowsGram) {  // a * conj(b)
                re += ar * br + ai * bi;
                im += ai * br - ar * bi;
            } else {         // conj(a) * b
                re += ar * br + ai * bi;
                im += ar * bi - ai * br;
            }
        }
        __syncthreads();
    }
    if (i < n && k < n) G[(size_t)k * n + i] = make_cuDoubleComplex(re, im);
}

cudaError_t dh_launch_gather_block(const float2* src0, const float2* src1, int pol0, int pol1, int polCount, int M,
                                   int rows, int batch, float2* A, cudaStream_t s) {
    const int total = rows * batch;
    int blocks = (total + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_gather_block<<<blocks, 256, 0, s>>>(src0, src1, pol0, pol1, polCount, M, rows, batch, A);
    return cudaGetLastError();
}

cudaError_t dh_launch_gram(const float2* A, int rows, int batch, int rowsGram, void* G, cudaStream_t s) {
    const int n = rowsGram ? rows : batch;
    dim3 grid((n + 15) / 16, (n + 15) / 16);
    k_gram<<<grid, dim3(16, 16), 0, s>>>(A, rows, batch, rowsGram, static_cast<cuDoubleComplex*>(G));
    return cudaGetLastError();
}
