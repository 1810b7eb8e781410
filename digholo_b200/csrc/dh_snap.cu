// Kernels of the AutoAlign parameter estimate ("snap", digHoloAutoAlignSnap
// digHolo.cpp:11517-11970, and digHoloAutoFocus digHolo.cpp:11181-11499).
// The snap looks at the whole polarisation half of each frame: FFT windows
// of (frameWidth / polCount) x frameHeight pixels, whose sides are multiples
// of 16 but rarely powers of two, so every transform here is a
// shared-memory mixed-radix FFT (radix 4 and 2, then the odd prime factors
// by direct DFT), FP32 with FP64-rounded twiddles:
//   * R2C planes of the frames' full windows (rows, then columns);
//   * batch-summed Fourier intensity (with and without the DC disk);
//   * the tilt correlation: FFTW REDFT10 (DCT-II) of the summed intensity,
//     the Gaussian filter (applied with the reference's flat indexing),
//     REDFT01 (DCT-III), in FP64 like the oracle's FFT library, and the
//     maximum outside the disk of radius 2 k0 aperture;
//   * the effective area of the summed intensity inside the Fourier window;
//   * reconstructed fields of the full window (the Fourier window with its
//     factors, placed as digHoloCopyWindow places it, inverse 2D FFT) and the
//     centre of mass and effective area of their summed intensity;
//   * the AutoFocus score: V = -conj(A . ref) with the 14-bit reference wave
//     of a trial defocus, inverse 2D FFT, effective area of the summed |.|^2.
// None of these kernels waits on another block or on a flag.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_snap.h"

using namespace dh;

namespace {

constexpr int ST = 256;            // threads per block
constexpr int SBUF = 8192;         // complex elements per shared transform buffer
constexpr int MAXP = 64;           // largest radix (odd prime factor) handled

// position of input n after the mixed-radix decimation-in-time permutation
__device__ __forceinline__ int mixPerm(int n, const DhMixPlan& pl) {
    int pos = 0, rem = n, size = pl.N;
    for (int s = pl.S - 1; s >= 0; s--) {
        const int p = pl.radix[s];
        size /= p;
        const int q = rem % p;
        rem /= p;
        pos += q * size;
    }
    return pos;
}

__device__ __forceinline__ float2 twAt(const float2* __restrict__ tw, int k, bool inv) {
    float2 w = __ldg(&tw[k]);
    if (inv) w.y = -w.y;
    return w;
}

// In-place mixed-radix DIT FFT of G vectors of length pl.N held contiguously
// in shared memory (vector v at buf + v N), input already permuted by
// mixPerm.  tw[k] = exp(-2 pi i k / N); inv selects exp(+2 pi i k / N)
// (unnormalised both ways).  Ends with a barrier.
__device__ void fftMixed(float2* buf, int G, const DhMixPlan& pl, const float2* __restrict__ tw, bool inv) {
    const int N = pl.N;
    int l = 1;
    for (int s = 0; s < pl.S; s++) {
        const int p = pl.radix[s], L = l * p, nb = N / p, tstride = N / L;
        for (int t = threadIdx.x; t < G * nb; t += blockDim.x) {
            const int v = t / nb, b = t - v * nb;
            const int g = b / l, j = b - g * l;
            float2* x = buf + (size_t)v * N + g * L + j;
            const int ts = j * tstride;
            if (p == 2) {
                const float2 a0 = x[0];
                const float2 a1 = cmul(x[l], twAt(tw, ts, inv));
                x[0] = cadd(a0, a1);
                x[l] = csub(a0, a1);
            } else if (p == 4) {
                const float2 a0 = x[0];
                const float2 a1 = cmul(x[l], twAt(tw, ts, inv));
                const float2 a2 = cmul(x[2 * l], twAt(tw, 2 * ts, inv));
                const float2 a3 = cmul(x[3 * l], twAt(tw, 3 * ts, inv));
                const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
                const float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
                // forward: -i d13; inverse: +i d13
                const float2 r = inv ? make_float2(-d13.y, d13.x) : make_float2(d13.y, -d13.x);
                x[0] = cadd(s02, s13);
                x[l] = cadd(d02, r);
                x[2 * l] = csub(s02, s13);
                x[3 * l] = csub(d02, r);
            } else {
                float2 a[MAXP];
                a[0] = x[0];
                for (int q = 1; q < p; q++) a[q] = cmul(x[q * l], twAt(tw, (q * ts) % N, inv));
                const int pstep = N / p;
                for (int qo = 0; qo < p; qo++) {
                    float2 acc = a[0];
                    for (int q = 1; q < p; q++) acc = cadd(acc, cmul(a[q], twAt(tw, ((q * qo) % p) * pstep, inv)));
                    x[qo * l] = acc;   // every input was read into a[] first
                }
            }
        }
        __syncthreads();
        l = L;
    }
}

// ---------------------------------------------------------------- Fourier planes

// G rows of one (frame, polarisation) full window: real row -> N = W point
// forward FFT -> columns 0 .. W/2 of the R2C plane [unit][H][W/2+1].
__global__ void __launch_bounds__(ST) k_snap_plane_rows(DhSnapPlaneArgs a) {
    extern __shared__ float2 sm[];
    const int W = a.W, H = a.H, Nx = W / 2 + 1, G = a.G;
    const int groups = (H + G - 1) / G;
    const int unit = blockIdx.x / groups, r0 = (blockIdx.x % groups) * G;
    const int P = a.polCount, pol = unit % P, frame = unit / P;
    const long long base = (long long)frame * a.frameStride + (long long)(a.cy[pol] + r0) * a.frameWidth + a.cx[pol];
    for (int e = threadIdx.x; e < G * W; e += blockDim.x) {
        const int v = e / W, n = e - v * W;
        float f = 0.f;
        if (r0 + v < H) {
            const long long o = base + (long long)v * a.frameWidth + n;
            f = a.u16 ? (float)static_cast<const unsigned short*>(a.frames)[o] : static_cast<const float*>(a.frames)[o];
        }
        sm[v * W + mixPerm(n, a.planW)] = make_float2(f, 0.f);
    }
    __syncthreads();
    fftMixed(sm, G, a.planW, a.twW, false);
    for (int e = threadIdx.x; e < G * Nx; e += blockDim.x) {
        const int v = e / Nx, k = e - v * Nx;
        if (r0 + v < H) a.plane[((size_t)unit * H + r0 + v) * Nx + k] = sm[v * W + k];
    }
}

// In-place (or out-of-place) FFT of `vecs` vectors of length N per unit:
// element e of vector v of unit u at u * unitStride + v * vecStride + e *
// elemStride.  Optional fused work: multiply by the separable 14-bit
// reference wave and take -conj before the transform (AutoFocus), or
// accumulate |.|^2 of the result into sum[pol][pixel] (atomic, per unit's
// polarisation) instead of storing it.
__global__ void __launch_bounds__(ST) k_snap_fft(DhSnapFftArgs a) {
    extern __shared__ float2 sm[];
    const int N = a.plan.N, G = a.G;
    const int groups = (a.vecs + G - 1) / G;
    const int unit = blockIdx.x / groups, v0 = (blockIdx.x % groups) * G;
    const float2* in = a.in + (size_t)unit * a.unitStride;
    float2* out = a.out + (size_t)unit * a.unitStride;
    const int pol = unit % a.polCount;
    const bool rowMajor = a.elemStride == 1;
    for (int t = threadIdx.x; t < G * N; t += blockDim.x) {
        int v, e;
        if (rowMajor) { v = t / N; e = t - v * N; }
        else { e = t / G; v = t - e * G; }
        float2 x = make_float2(0.f, 0.f);
        if (v0 + v < a.vecs) {
            const size_t off = (size_t)(v0 + v) * a.vecStride + (size_t)e * a.elemStride;
            x = in[off];
            if (a.ref) {
                // pixel (y, x) of the field: rows are vectors here
                const int px = e, py = v0 + v;
                const short* rw = a.ref + (size_t)pol * 2 * (a.nx + a.ny);
                const int xr = rw[px], xi = rw[a.nx + px];
                const int yr = rw[2 * a.nx + py], yi = rw[2 * a.nx + a.ny + py];
                const float k = 1.0f / (16383.0f * 16383.0f);
                const float adjR = k * (float)(yr * xr - yi * xi);
                const float adjI = k * (float)(yr * xi + yi * xr);
                // applyTilt16 (digHolo.cpp:2781-2797): V = -conj(A adj)
                x = make_float2(x.y * adjI - x.x * adjR, x.x * adjI + x.y * adjR);
            }
        }
        sm[v * N + mixPerm(e, a.plan)] = x;
    }
    __syncthreads();
    fftMixed(sm, G, a.plan, a.tw, a.inverse != 0);
    for (int t = threadIdx.x; t < G * N; t += blockDim.x) {
        int v, e;
        if (rowMajor) { v = t / N; e = t - v * N; }
        else { e = t / G; v = t - e * G; }
        if (v0 + v >= a.vecs) continue;
        const float2 y = sm[v * N + e];
        const size_t off = (size_t)(v0 + v) * a.vecStride + (size_t)e * a.elemStride;
        if (a.sum) atomicAdd(&a.sum[(size_t)pol * a.sumStride + off], fmaf(y.x, y.x, y.y * y.y));
        else out[off] = y;
    }
}

// Batch-summed normalised intensity of the planes per pixel, in frame
// order (as the reference accumulates it), zero outside the analysed
// region: rows 0 and H/2, column 0 and columns from 8 floor(Nx/8) on, and,
// when r2 > 0, the DC disk kx^2 + ky^2 < r2.
__global__ void k_snap_batchsum(const float2* __restrict__ plane, int frames, int P, int H, int Nx,
                                const float* __restrict__ kx, const float* __restrict__ ky, float r2, float* sum) {
    const float norm = (float)(1.0 / ((double)Nx * (double)H));
    const int nxr = 8 * (Nx / 8);
    const int total = P * H * Nx;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int pol = e / (H * Nx), pix = e - pol * H * Nx;
        const int j = pix / Nx, i = pix - j * Nx;
        bool in = !(j == 0 || j == H / 2 || i == 0 || i >= nxr);
        if (in && r2 > 0.f) in = __fadd_rn(__fmul_rn(kx[i], kx[i]), __fmul_rn(ky[j], ky[j])) >= r2;
        float acc = 0.f;
        if (in) {
            for (int b = 0; b < frames; b++) {
                const float2 v = plane[((size_t)b * P + pol) * H * Nx + pix];
                acc += fmaf(v.x, v.x, v.y * v.y) * norm;
            }
        }
        sum[(size_t)pol * H * Nx + pix] = acc;
    }
}

// ---------------------------------------------------------------- tilt correlation

// One 1D pass of FFTW's REDFT10 (kind 2) or REDFT01 (kind 3) over an
// n0 x n1 array, along axis 1 (rows, length n1) or axis 0 (columns, length
// n0), FP64; the input is float or double, the output double or float.
__global__ void k_snap_dct(const float* inF, const double* inD, double* outD, float* outF, int n0, int n1, int axis,
                           int kind, const double* __restrict__ cosTab) {
    const int n = axis == 1 ? n1 : n0;
    const int period = 4 * n;
    const int total = n0 * n1;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int r = e / n1, c = e - r * n1;
        const int k = axis == 1 ? c : r;
        auto at = [&](int j) -> double {
            const size_t o = axis == 1 ? (size_t)r * n1 + j : (size_t)j * n1 + c;
            return inF ? (double)inF[o] : inD[o];
        };
        double acc;
        if (kind == 2) {
            acc = 0.0;
            for (int j = 0; j < n; j++) acc += at(j) * cosTab[((2 * j + 1) * k) % period];
            acc *= 2.0;
        } else {
            double s = 0.0;
            for (int j = 1; j < n; j++) s += at(j) * cosTab[(j * (2 * k + 1)) % period];
            acc = at(0) + 2.0 * s;
        }
        if (outD) outD[e] = acc;
        else outF[e] = (float)acc;
    }
}

// The Gaussian filter of the correlation with the reference's indexing
// (digHolo.cpp:11611-11643): the (H, Nx) array is walked in blocks of 8
// floats, 8 floor(Nx/8) floats per row index, without the row stride, so
// flat position f gets the factor of row f / (8 floor(Nx/8)) and column
// f mod (8 floor(Nx/8)); the last H floats keep their values.
__global__ void k_snap_filter(float* a, int H, int Nx, float wx2, float wy2, float ps, float ps2) {
    const int nb = 8 * (Nx / 8);
    const int total = H * nb;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        const int j = f / nb, i = f - j * nb;
        const float x = __fmul_rn((float)i, ps);
        const float xw2 = __fmul_rn(__fmul_rn(x, x), wx2);
        const float y2 = __fmul_rn((float)(j * j), ps2);
        const float yw2 = __fmul_rn(y2, wy2);
        a[f] = __fmul_rn(a[f], expf(__fadd_rn(xw2, yw2)));
    }
}

// Position of the maximum of the correlation among pixels with
// kx^2 + ky^2 > ad (the first in row-major order on ties), per
// polarisation plane; out[pol] = flat index j Nx + i, or -1.
__global__ void __launch_bounds__(ST) k_snap_argmax(const float* __restrict__ a, int H, int Nx,
                                                    const float* __restrict__ kx, const float* __restrict__ ky,
                                                    float ad, size_t planeStride, int* out) {
    const float* pl = a + (size_t)blockIdx.x * planeStride;
    float best = -INFINITY;
    int bi = -1;
    for (int e = threadIdx.x; e < H * Nx; e += blockDim.x) {
        const int j = e / Nx, i = e - j * Nx;
        const float kr = __fadd_rn(__fmul_rn(kx[i], kx[i]), __fmul_rn(ky[j], ky[j]));
        if (!(kr > ad)) continue;
        const float v = pl[e];
        if (v > best || (v == best && (bi < 0 || e < bi))) { best = v; bi = e; }
    }
    __shared__ float sv[ST];
    __shared__ int si[ST];
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = ST / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const float v = sv[threadIdx.x + s];
            const int i2 = si[threadIdx.x + s];
            if (i2 >= 0 && (si[threadIdx.x] < 0 || v > sv[threadIdx.x] || (v == sv[threadIdx.x] && i2 < si[threadIdx.x]))) {
                sv[threadIdx.x] = v;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = si[0];
}

// Sums over one plane per block (FP64): out[pol][4] = {sum S, sum x S,
// sum y S, sum S^2} where S is the plane, masked for the windowed Fourier
// analysis when `window` is set (rows 0 and H/2, column 0 and the columns
// from 8 floor(Nx/8) on excluded, (kx - cx)^2 + (ky - cy)^2 <= w2).
__global__ void __launch_bounds__(ST) k_snap_moments(const float* __restrict__ S, int ny, int nx, size_t planeStride,
                                                     const float* __restrict__ xa, const float* __restrict__ ya,
                                                     int window, const float* __restrict__ cxy, float w2,
                                                     double* out) {
    const int pol = blockIdx.x;
    const float* pl = S + (size_t)pol * planeStride;
    const int nxr = 8 * (nx / 8);
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    for (int e = threadIdx.x; e < ny * nx; e += blockDim.x) {
        const int j = e / nx, i = e - j * nx;
        if (window) {
            if (j == 0 || j == ny / 2 || i == 0 || i >= nxr) continue;
            const float dx = __fsub_rn(xa[i], cxy[2 * pol]);
            const float dy = __fsub_rn(ya[j], cxy[2 * pol + 1]);
            if (!(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) <= w2)) continue;
        }
        const double v = pl[e];
        m[0] += v;
        m[1] += (double)xa[i] * v;
        m[2] += (double)ya[j] * v;
        m[3] += v * v;
    }
    __shared__ double red[4][ST];
    for (int q = 0; q < 4; q++) red[q][threadIdx.x] = m[q];
    __syncthreads();
    for (int s = ST / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 4; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) out[pol * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// ---------------------------------------------------------------- reconstructed fields

// The Fourier window of each (frame, polarisation) with its factors, placed
// as digHoloCopyWindow places it (digHolo.cpp:1808-2122): at the origin of
// an h x w field (low resolution), or at row (j + SY + H/2) mod H and column
// (SX - W/2 + c) mod W of an H x W field, zero elsewhere (full resolution).
__global__ void k_snap_place(DhSnapPlaceArgs a) {
    const int W = a.W, H = a.H, Nx = W / 2 + 1, w = a.w, h = a.h;
    const int P = a.polCount;
    const size_t fieldN = (size_t)a.ny * a.nx;
    const size_t total = (size_t)a.units * fieldN;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int unit = (int)(e / fieldN);
        const int pix = (int)(e - (size_t)unit * fieldN);
        const int pol = unit % P;
        const int y = pix / a.nx, x = pix - y * a.nx;
        int j, c;
        if (a.lowres) {
            j = y;
            c = x;
        } else {
            // invert the placement: row = (j + SY + H/2) mod H, col = (sx0 + c) mod W
            j = ((y - a.SY[pol] - H / 2) % H + H) % H;
            c = ((x - a.sx0[pol]) % W + W) % W;
        }
        float2 v = make_float2(0.f, 0.f);
        if (j < h && c < w) {
            const int row = ((j + a.SY[pol] + H / 2) % H + H) % H;
            const int col = a.sx0[pol] + c;
            if (col >= 0 && col < Nx) {
                v = cmul(a.plane[((size_t)unit * H + row) * Nx + col], a.adj[((size_t)pol * h + j) * w + c]);
            }
        }
        a.field[e] = v;
    }
}

// Batch-summed |E|^2 / (nx ny) of the fields per pixel, in frame order.
__global__ void k_snap_field_sum(const float2* __restrict__ f, int frames, int P, size_t n, float norm, float* sum) {
    const size_t total = (size_t)P * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int pol = (int)(e / n);
        const size_t pix = e - (size_t)pol * n;
        float acc = 0.f;
        for (int b = 0; b < frames; b++) {
            const float2 v = f[((size_t)b * P + pol) * n + pix];
            acc += fmaf(v.x, v.x, v.y * v.y) * norm;
        }
        sum[e] = acc;
    }
}

int gridFor(size_t total) {
    size_t g = (total + ST - 1) / ST;
    const size_t cap = (size_t)smCountCached() * 16;
    return (int)(g < cap ? (g ? g : 1) : cap);
}

}  // namespace

// Radices for a transform of length N: 4s, a 2, then odd primes; false when
// a prime factor exceeds the largest radix handled.
bool dh_mix_plan(int N, DhMixPlan& pl) {
    pl.N = N;
    pl.S = 0;
    int m = N;
    while (m % 4 == 0 && pl.S < 24) { pl.radix[pl.S++] = 4; m /= 4; }
    while (m % 2 == 0 && pl.S < 24) { pl.radix[pl.S++] = 2; m /= 2; }
    for (int p = 3; m > 1 && pl.S < 24; p += 2) {
        while (m % p == 0 && pl.S < 24) {
            if (p > MAXP) return false;
            pl.radix[pl.S++] = p;
            m /= p;
        }
    }
    return m == 1 && N >= 1;
}

int dh_snap_vectors_per_block(int N) { return N <= SBUF ? SBUF / N : 0; }

cudaError_t dh_launch_snap_plane_rows(const DhSnapPlaneArgs& a, cudaStream_t s) {
    if (a.G < 1 || a.G * a.W > SBUF) return cudaErrorNotSupported;
    const size_t smem = sizeof(float2) * (size_t)a.G * a.W;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_snap_plane_rows), (int)(sizeof(float2) * SBUF));
    if (e != cudaSuccess) return e;
    const int groups = (a.H + a.G - 1) / a.G;
    k_snap_plane_rows<<<(unsigned)(a.units * groups), ST, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_fft(const DhSnapFftArgs& a, cudaStream_t s) {
    if (a.G < 1 || a.G * a.plan.N > SBUF) return cudaErrorNotSupported;
    const size_t smem = sizeof(float2) * (size_t)a.G * a.plan.N;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_snap_fft), (int)(sizeof(float2) * SBUF));
    if (e != cudaSuccess) return e;
    const int groups = (a.vecs + a.G - 1) / a.G;
    k_snap_fft<<<(unsigned)(a.units * groups), ST, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_batchsum(const float2* plane, int frames, int P, int H, int Nx, const float* kx,
                                    const float* ky, float r2, float* sum, cudaStream_t s) {
    k_snap_batchsum<<<gridFor((size_t)P * H * Nx), ST, 0, s>>>(plane, frames, P, H, Nx, kx, ky, r2, sum);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_dct(const float* inF, const double* inD, double* outD, float* outF, int n0, int n1,
                               int axis, int kind, const double* cosTab, cudaStream_t s) {
    k_snap_dct<<<gridFor((size_t)n0 * n1), ST, 0, s>>>(inF, inD, outD, outF, n0, n1, axis, kind, cosTab);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_filter(float* a, int H, int Nx, float wx2, float wy2, float ps, float ps2, cudaStream_t s) {
    k_snap_filter<<<gridFor((size_t)H * Nx), ST, 0, s>>>(a, H, Nx, wx2, wy2, ps, ps2);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_argmax(const float* a, int planes, int H, int Nx, const float* kx, const float* ky, float ad,
                                  size_t planeStride, int* out, cudaStream_t s) {
    k_snap_argmax<<<planes, ST, 0, s>>>(a, H, Nx, kx, ky, ad, planeStride, out);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_moments(const float* S, int planes, int ny, int nx, size_t planeStride, const float* xa,
                                   const float* ya, int window, const float* cxy, float w2, double* out, cudaStream_t s) {
    k_snap_moments<<<planes, ST, 0, s>>>(S, ny, nx, planeStride, xa, ya, window, cxy, w2, out);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_place(const DhSnapPlaceArgs& a, cudaStream_t s) {
    k_snap_place<<<gridFor((size_t)a.units * a.nx * a.ny), ST, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t dh_launch_snap_field_sum(const float2* f, int frames, int P, size_t n, float norm, float* sum,
                                     cudaStream_t s) {
    k_snap_field_sum<<<gridFor((size_t)P * n), ST, 0, s>>>(f, frames, P, n, norm, sum);
    return cudaGetLastError();
}
