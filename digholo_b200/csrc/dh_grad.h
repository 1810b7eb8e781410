// Launch parameters of the adjoint kernels (dh_align_grad.cu) shared with
// the host optimiser (dh_align_adjoint.cpp).
#pragma once
#include <cuda_runtime.h>

struct DhGradParams {
    const float2* V;        // [unit][ny][nx]  -conj(A R)
    const float2* Vx;       // [unit][ny][nx]  -conj(A_x R)
    const float2* Vy;       // [unit][ny][nx]  -conj(A_y R)
    const float2* coefs;    // [frame][pol * M + mode]
    const float* hx;        // [pol][G + 2][nx] float modes (unquantised)
    const float* hy;        // [pol][G + 2][ny]
    const float* xAxis;     // [nx]
    const float* yAxis;     // [ny]
    int nx, ny, frameCount, polCount, G, M;
    float k0u[2];           // k0 * pi / 180 (per polarisation: the same)
    float tiltX[2], tiltY[2];   // degrees (the values the reference wave of this polarisation uses)
    float bcx[2], bcy[2];       // beam centre (m) of this polarisation
    float piOverLambda;
    float waist[2];
    float* out;             // [unit][7]: tx, ty, defocus, bcx, bcy, waist, sum |c|^2
    // optional weights [frame][pol * M + mode] in place of conj(c): the
    // kernel then returns Re sum w dc (the MDL gradient's contraction)
    const float2* weights;
};

// Per field only the captured power sum |c|^2 into out[unit * 7 + 6] (the
// other six entries zero), summed in the order of the gradient kernels, so
// the value equals theirs bit for bit: the value of a line-search trial.
cudaError_t dh_launch_align_power(const DhGradParams& p, cudaStream_t s);

cudaError_t dh_launch_window_deriv(const float2* W, const float* kxw, const float* kyw, int w, int h, int polCount, int units,
                                   float2* Wx, float2* Wy, cudaStream_t s);
cudaError_t dh_launch_align_grad(const DhGradParams& p, cudaStream_t s);
cudaError_t dh_launch_mdl_weights(const float2* A, int rows, int batch, int rowsGram, const double2* u, double alpha,
                                  int pol0, int pol1, int polCount, int M, float2* W, cudaStream_t s);
