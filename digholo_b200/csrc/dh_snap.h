// Argument blocks and launchers of the AutoAlign parameter-estimate kernels
// (dh_snap.cu), shared with the host logic (dh_snap.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

// Mixed-radix transform plan: N = radix[0] * ... * radix[S-1].
struct DhMixPlan {
    int N;
    int S;
    int radix[24];
};

// R2C rows of the frames' full windows.
struct DhSnapPlaneArgs {
    const void* frames;
    int u16;
    int frameWidth;
    long long frameStride;      // elements between frames
    int cx[2], cy[2];           // window corners per polarisation
    int W, H, polCount, units;  // units = frames * polCount
    int G;                      // rows per block
    DhMixPlan planW;
    const float2* twW;          // exp(-2 pi i k / W), k < W
    float2* plane;              // out: [unit][H][W/2+1]
};

// Batched 1D FFT along one axis (see k_snap_fft).
struct DhSnapFftArgs {
    const float2* in;
    float2* out;
    size_t unitStride;          // elements between units
    int units, vecs;            // units, vectors per unit
    size_t vecStride, elemStride;
    int G;                      // vectors per block
    int inverse;
    DhMixPlan plan;
    const float2* tw;           // exp(-2 pi i k / N), k < N
    int polCount;               // unit u belongs to polarisation u % polCount
    // optional: -conj(x . ref) before the transform (row pass of a field)
    const short* ref;           // [pol][Xr(nx) Xi(nx) Yr(ny) Yi(ny)] 14-bit
    int nx, ny;
    // optional: accumulate |y|^2 into sum[pol * sumStride + pixel] instead of storing y
    float* sum;
    size_t sumStride;
};

// Fourier windows placed into field planes (see k_snap_place).
struct DhSnapPlaceArgs {
    const float2* plane;        // [unit][H][W/2+1]
    const float2* adj;          // [pol][h][w] window factors
    float2* field;              // out: [unit][ny][nx]
    int W, H, w, h, nx, ny, lowres, polCount, units;
    int sx0[2], SY[2];
};

bool dh_mix_plan(int N, DhMixPlan& pl);
int dh_snap_vectors_per_block(int N);
cudaError_t dh_launch_snap_plane_rows(const DhSnapPlaneArgs& a, cudaStream_t s);
cudaError_t dh_launch_snap_fft(const DhSnapFftArgs& a, cudaStream_t s);
cudaError_t dh_launch_snap_batchsum(const float2* plane, int frames, int P, int H, int Nx, const float* kx,
                                    const float* ky, float r2, float* sum, cudaStream_t s);
cudaError_t dh_launch_snap_dct(const float* inF, const double* inD, double* outD, float* outF, int n0, int n1,
                               int axis, int kind, const double* cosTab, cudaStream_t s);
cudaError_t dh_launch_snap_filter(float* a, int H, int Nx, float wx2, float wy2, float ps, float ps2, cudaStream_t s);
cudaError_t dh_launch_snap_argmax(const float* a, int planes, int H, int Nx, const float* kx, const float* ky, float ad,
                                  size_t planeStride, int* out, cudaStream_t s);
cudaError_t dh_launch_snap_moments(const float* S, int planes, int ny, int nx, size_t planeStride, const float* xa,
                                   const float* ya, int window, const float* cxy, float w2, double* out, cudaStream_t s);
cudaError_t dh_launch_snap_place(const DhSnapPlaceArgs& a, cudaStream_t s);
cudaError_t dh_launch_snap_field_sum(const float2* f, int frames, int P, size_t n, float norm, float* sum,
                                     cudaStream_t s);
