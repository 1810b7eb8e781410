// Launch parameters shared by the host runtime (dh_runtime.cpp) and the
// kernels (dh_kernels.cu).  Plain structs, passed by value to kernels.
#pragma once
#include <stdint.h>

#define DH_MAXPOL 2

// Forward stage: frame window -> pruned R2C FFT -> Fourier window with the
// reference's window operations (digHolo.cpp:6986-7260 and 1808-2122).
struct DhFwdParams {
    const void* frames;     // device pointer to the batch, uint16 or float32
    int inputU16;           // 1: uint16 pixels, 0: float32 pixels
    int frameWidth;         // pixels per frame row
    long long frameStride;  // pixels between frames
    int frameCount;         // frames to process (batchCount * avgCount)
    int polCount;
    int logW, logH;         // FFT window is 2^logW x 2^logH
    int cx[DH_MAXPOL], cy[DH_MAXPOL];   // FFT window corner in the frame
    int w, h;               // IFFT window size
    int colChunk;           // columns of the IFFT window handled per block (divides w)
    int sx0[DH_MAXPOL];     // first kx column of the IFFT window (SX - W/2)
    int sy[DH_MAXPOL];      // SY (row origin in fftshifted coordinates)
    float bcx[DH_MAXPOL], bcy[DH_MAXPOL];   // beam centre relative to FFT window centre (m)
    float kx0[DH_MAXPOL], ky0[DH_MAXPOL];   // window centre k0*sin(tilt)
    float r02[DH_MAXPOL];                   // (k0*sin(radius))^2
    float kyShift;          // |dky * H|, the unwrapped-row offset for the mask
    float norm;             // 1/sqrt(W*H*ifftLength)
    float halfPixel;        // pixelSize / 2
    int fillFactor;         // apply x/sin(x) in kx and ky
    const float* kxAxis;    // fftshifted kx axis (W)
    const float* kyAxis;    // fftshifted ky axis (H)
    const float2* batchCal; // optional per-frame complex factor [pol][batchCalCount]
    int batchCalCount;
    int frameOffset;        // index of frame 0 of this launch within the batch
    float2* window;         // out: [frame][pol][h][w]
    const float2* twiddle;  // TW_N twiddles
    // Frame-independent factors, precomputed per configuration for the
    // register kernel (the generic kernel evaluates them itself):
    const float2* tabSplit; // [pol][w]    exp(-2 pi i (sx0 + c) / W), the R2C split twiddles
    const float2* tabCol;   // [pol][h][Q] exp(-2 pi i row_j b / H), Q = H / h
    const float2* tabAdj;   // [pol][h][w] mask x norm x 1/sinc x exp(i (kx bcx + ky bcy))
    // Tensor-core row DFT of uint16 frames: 22-bit fixed-point (cos + 1,
    // -sin + 1) of the kept kx columns plus a ones column, as byte digits in
    // the swizzled K-major operand layout [pol][4][2W / 128][dftNpad][128 B].
    const unsigned char* dftDigits;
    int dftNpad;
    int* status;            // set to 1 by a kernel whose bounded wait expired (host-mapped)
};

// Inverse stage: Fourier window -> IFFT -> field statistics -> reference wave,
// -conj, int16 rounding -> separable HG overlap
// (digHolo.cpp:8558-8760, 8788-9341, 9353-9815).
struct DhInvParams {
    const float2* window;   // [frame][pol][h][w]
    int frameCount, polCount;
    int lowres;             // 1: field is h x w, 0: field is H x W
    int logW, logH;         // FFT window (full-res field) sizes
    int logw, logh;         // IFFT window sizes (ceil log2; exact for power-of-two windows)
    int w, h;               // IFFT window sides (multiples of 16)
    int sx0[DH_MAXPOL];     // kx column of window column 0 (full-res placement)
    int sy[DH_MAXPOL];      // row origin for full-res placement
    const short* refWave;   // [pol][2*(nx+ny)]: Xr, Xi, Yr, Yi (14-bit ints)
    const float* refWaveF;  // [pol][2*(nx+ny)]: the same wave unquantised, for field32
    const float* xAxis;     // reconstructed-plane axes (nx, ny)
    const float* yAxis;
    float dA;               // pixel area of the reconstructed plane
    short* fieldR;          // out: [frame][pol][ny][nx]
    short* fieldI;
    float2* field32;        // optional out: float field -conj(A.ref) before rounding
    float* stats;           // out: [param][pol][frameCount+1] (DIGHOLO_ANALYSIS layout)
    int statsStride;        // frameCount+1 entries per (param, pol)
    // overlap
    int maxMG;              // 0: no overlap
    int modeCount;
    const short* hgX;       // [pol][maxMG][nx] int16 modes
    const short* hgY;       // [pol][maxMG][ny]
    const float* hgScaleX;  // [pol][maxMG]
    const float* hgScaleY;
    float2* coefs;          // out: [frame][pol*modeCount + mode]
    const float2* twiddle;
    int* status;            // set by a kernel whose bounded wait expired (host-mapped)
    // optional reference-wave calibration [pol][ny][nx]: multiplies the IFFT
    // output before the statistics and the tilt removal (block-per-unit kernels)
    const float2* refCal;
    // 1: only field32 is wanted (the adjoint's derivative fields); kernels
    // that honour it skip the int16 planes (fieldR, fieldI are then unused)
    int fieldsOnly;
};

// Separable DFT stage of the calibration planes: out[u][a][b] =
// sum_k in[u inU + a inA + b inB + k inK] exp(sign 2 pi i fo fk / N), fo the
// frequency of the output index (a or b), fk that of k (each an index table
// per polarisation u % fP, or the index itself), accumulated in FP64 and
// rounded to FP32; then optionally times ufac[u] (complex) and fac[u % fP][a][b].
struct DhCalDft {
    const float2* in;
    long long inU, inA, inB, inK;
    float2* out;            // dense [U][A][B]
    int U, A, B, K;
    const int* freqOut;     // [fP][A or B] or null
    int outOnA;             // 1: freqOut indexes a, 0: b
    const int* freqK;       // [fP][K] or null
    int fP;                 // period of u for the per-polarisation tables (>= 1)
    int N;                  // transform length (<= 4096; frequencies are non-negative)
    int sign;               // -1 forward, +1 inverse
    const float2* ufac;     // [U] or null
    const float* fac;       // [fP][A][B] or null
};

// FP64 Hermite-Gaussian basis along one axis (digHolo.cpp:1269-1484).
struct DhBasisParams {
    const float* axis;   // float axis values
    int count;           // samples
    int modes;           // maxMG
    double w0;
    short* out16;        // [modes][count]
    float* scale;        // [modes] float value of one int16 step
    float* outF;         // optional [modes][count] unquantised float modes
    int modes16;         // modes written to out16 / scale (the first modes16)
};

// Full R2C Fourier planes of the FFT windows and their analysis (the
// reference's digHoloPixelsFourierPlane and digHoloFFTAnalysis).
struct DhFourierParams {
    DhFwdParams f;          // frame source and FFT-window geometry
    float2* plane;          // out: [frame][pol][H][W/2+1]
    const float* kx;        // fftshifted kx axis (W)
    const float* ky;        // fftshifted ky axis (H)
    float r2;               // squared radius of the excluded disk (0: none)
    float* stats;           // out: [param][pol][frameCount + 1] (DIGHOLO_ANALYSIS layout)
    float* batchSum;        // out: [pol][W H], pixel (j, i) at j (W/2+1) + i
    int windowCols;         // 1: column transforms of each polarisation's Fourier-window columns only
};
