// Argument blocks and launchers of the frame simulator kernels (dh_sim.cu),
// shared with its host logic (dh_sim.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

// One term of a polarisation region's field: coefficient c xScale yScale as
// float, column mode m, row mode n.
struct DhSimMode {
    float cr, ci;
    int m, n;
};

struct DhSimFieldArgs {
    const DhSimMode* modes;     // the terms of every (frame, pol), in mode order
    const int* modeOffset;      // [frames * polCount + 1] start of each unit's terms
    const short* hgCol;         // [pol][G][cols] int16 modes along the region's columns
    const short* hgRow;         // [pol][G][rows] int16 modes along the rows
    const float2* refCol;       // [pol][cols] reference wave factor along the columns
    const float2* refRow;       // [pol][rows] factor along the rows
    float* out;                 // [frame][rows][frameWidth] intensity
    unsigned* maxBits;          // running maximum of the intensity (float bits)
    int frames, polCount, rows, cols, frameWidth, G;
};

cudaError_t dh_launch_sim_field(const DhSimFieldArgs& a, int maxModesPerUnit, cudaStream_t s);
// Basis fields: frames = output modes, out [mode][pol][rows][cols] complex.
cudaError_t dh_launch_basis_fields(const DhSimFieldArgs& a, int maxModesPerUnit, float2* out, cudaStream_t s);
cudaError_t dh_launch_sim_sinc(float2* X, int frames, int H, int Nx, const float* sincX, const float* sincY, float norm,
                               cudaStream_t s);
cudaError_t dh_launch_sim_extend(const float2* half, float2* full, int frames, int H, int W, cudaStream_t s);
cudaError_t dh_launch_sim_real(const float2* full, float* out, size_t n, cudaStream_t s);
cudaError_t dh_launch_sim_quant(float* frames, unsigned short* frames16, size_t n, const unsigned* maxBits, int levels,
                                cudaStream_t s);
