// Forward stage of 512-pixel-wide FFT windows (the large-field workload:
// 2048x2048 frames, 512x512 windows, 64x64 IFFT windows) without the full
// Fourier plane: the same results as k_fourier_rows + k_fourier_cols +
// k_window_from_plane (dh_fourier.cu), i.e. the reference's FFTW r2c of the
// window (digHolo.cpp:7184-7260) and digHoloCopyWindow (digHolo.cpp:1808-2122),
// to FP32 rounding.
//
// k_plane_rows512: 16 rows per block, 16 threads per row.  The real row of
// 512 pixels is the complex sequence z[n] = f[2n] + i f[2n+1] of 256 points,
// transformed as 16 x 16 in registers: each thread takes z[16 n1 + t], a
// 16-point DFT over n1, the twiddle exp(-2 pi i t k1 / 256), one exchange
// through the row's own shared buffer (XOR-swizzled, warp barriers only), a
// 16-point DFT over n2; then the R2C
// split of the kept kx columns only.  Frame rows arrive by 16-byte loads.
//
// k_plane_window64: the column stage for 64x64 IFFT windows, only the 64
// kept ky rows: with H = Q 64 rows, X[k] = sum_b exp(-2 pi i b k / H)
// Z_b[k mod 64], Z_b the 64-point DFT of the decimated column x[Q a + b]
// (8 x 8 in registers, eight threads per transform); then the window
// factors (mask, normalisation, inverse pixel sinc, beam-centre phase) and
// the batch calibration.  Eight columns of one (frame, polarisation) per
// block, 512 threads.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"

using namespace dh;

namespace {

// cos and sin of 2 pi m / 16, m = 0..9
__device__ __constant__ float kC16[10] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                                          -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f, -1.0f,
                                          -0.92387953251128674f};
__device__ __constant__ float kS16[10] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f, 1.0f,
                                          0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                                          -0.38268343236508977f};

// 4-point DFT in place, natural order; exp(-2 pi i / 4) (or + for inverse)
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    const float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
    const float2 r = make_float2(d13.y, -d13.x);   // -i d13
    a0 = cadd(s02, s13);
    a1 = cadd(d02, r);
    a2 = csub(s02, s13);
    a3 = csub(d02, r);
}

// 16-point forward DFT in registers: input v[n] natural; output X[k] at
// v[4 (k mod 4) + k / 4] (n = 4 n1 + n2, k = k1 + 4 k2).
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
#pragma unroll
    for (int k1 = 1; k1 < 4; k1++) {
#pragma unroll
        for (int n2 = 1; n2 < 4; n2++) {
            const int m = n2 * k1;
            v[4 * k1 + n2] = cmul(v[4 * k1 + n2], make_float2(kC16[m], -kS16[m]));
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
}

__device__ __forceinline__ float2 at16(const float2 (&v)[16], int k) { return v[4 * (k & 3) + (k >> 2)]; }

// 8-point forward DFT in registers, natural order in and out.
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4(e0, e1, e2, e3);
    dft4(o0, o1, o2, o3);
    const float r = 0.70710678118654752f;
    const float2 t1 = cmul(o1, make_float2(r, -r));
    const float2 t2 = make_float2(o2.y, -o2.x);
    const float2 t3 = cmul(o3, make_float2(-r, -r));
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1);
    v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2);
    v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3);
    v[7] = csub(e3, t3);
}

constexpr int RR = 16;           // rows per block
constexpr int RN = 256;          // complex points per row (W = 512)

constexpr int NG = 4;            // row groups per block, the next one's pixels prefetched into registers

// Loads of row group g (16 rows of one unit): 16-byte loads, 8 uint16 or 4
// float pixels each, into registers.
template <bool U16>
struct RowRaw {
    static constexpr int N = U16 ? 4 : 8;
    uint4 u[N];
    __device__ __forceinline__ void load(const DhFwdParams& f, int unit, int r0, int tid) {
        const int P = f.polCount, pol = unit % P, frame = unit / P;
        const long long base = (long long)frame * f.frameStride + (long long)(f.cy[pol] + r0) * f.frameWidth + f.cx[pol];
        const int es = U16 ? 2 : 4;
        const unsigned char* fr = static_cast<const unsigned char*>(f.frames) + base * es;
#pragma unroll
        for (int i = 0; i < N; i++) {
            const int e = tid + 256 * i, rr = e / (N * 16), c = e % (N * 16);
            u[i] = __ldg(reinterpret_cast<const uint4*>(fr + ((long long)rr * f.frameWidth) * es + 16 * c));
        }
    }
    // as complex pairs z[n] = f[2n] + i f[2n + 1] into rows of RN
    __device__ __forceinline__ void store(float2* A, int tid) const {
#pragma unroll
        for (int i = 0; i < N; i++) {
            const int e = tid + 256 * i, rr = e / (N * 16), c = e % (N * 16);
            if (U16) {
                float4* d = reinterpret_cast<float4*>(A + rr * RN + 4 * c);
                d[0] = make_float4((float)(u[i].x & 0xFFFFu), (float)(u[i].x >> 16), (float)(u[i].y & 0xFFFFu),
                                   (float)(u[i].y >> 16));
                d[1] = make_float4((float)(u[i].z & 0xFFFFu), (float)(u[i].z >> 16), (float)(u[i].w & 0xFFFFu),
                                   (float)(u[i].w >> 16));
            } else {
                *reinterpret_cast<uint4*>(A + rr * RN + 2 * c) = u[i];
            }
        }
    }
};

// compact = 1: the kept columns only, rows of w values ([unit][H][w]);
// compact = 0: the plane's layout ([unit][H][W/2 + 1]).  A block takes NG
// consecutive groups of 16 rows.  A row's 16 threads are 16 lanes of one
// warp, so its exchange needs only warp barriers; the exchange reuses the
// row's buffer, value (k1, t) at 16 k1 + (t ^ k1).
template <bool U16>
__global__ void __launch_bounds__(256, U16 ? 4 : 3) k_plane_rows512(DhFourierParams q, int compact) {
    extern __shared__ float2 sp[];
    float2* A = sp;                          // [RR][RN] z, the exchange, then X
    const DhFwdParams& f = q.f;
    const int H = 1 << f.logH, Nx = RN + 1;
    const int groups = H / RR;
    const int total = f.frameCount * f.polCount * groups;
    const int g0 = blockIdx.x * NG;
    const int tid = threadIdx.x;
    const int r = tid >> 4, t = tid & 15;
    float2* Ar = A + r * RN;
    RowRaw<U16> raw;
    raw.load(f, g0 / groups, (g0 % groups) * RR, tid);
    for (int gi = 0; gi < NG; gi++) {
        const int g = g0 + gi;
        if (g >= total) break;
        const int unit = g / groups, r0 = (g % groups) * RR;
        const int pol = unit % f.polCount;
        __syncthreads();   // the previous group's split has read A
        raw.store(A, tid);
        if (gi + 1 < NG && g + 1 < total) raw.load(f, (g + 1) / groups, ((g + 1) % groups) * RR, tid);
        __syncthreads();
        float2 v[16];
        // first pass: n = 16 n1 + t, DFT over n1, twiddle exp(-2 pi i t k1 / 256)
#pragma unroll
        for (int n1 = 0; n1 < 16; n1++) v[n1] = Ar[16 * n1 + t];
        dft16(v);
        __syncwarp();
#pragma unroll
        for (int k1 = 0; k1 < 16; k1++) {
            float2 y = at16(v, k1);
            if (k1 && t) y = cmul(y, __ldg(&f.twiddle[(t * k1) << (TW_LOG - 8)]));
            Ar[16 * k1 + (t ^ k1)] = y;
        }
        __syncwarp();
        // second pass: thread t now holds k1 = t, DFT over n2; X[t + 16 k2]
#pragma unroll
        for (int n2 = 0; n2 < 16; n2++) v[n2] = Ar[16 * t + (n2 ^ t)];
        dft16(v);
        __syncwarp();
#pragma unroll
        for (int k2 = 0; k2 < 16; k2++) Ar[t + 16 * k2] = at16(v, k2);
        __syncthreads();
        // R2C split of the kept columns: F[k] = (Z[k] + conj Z[N-k]) / 2 - i e^{-2 pi i k / 512} (Z[k] - conj Z[N-k]) / 2
        const int kcount = q.windowCols ? f.w : Nx;
        const int kbeg = q.windowCols ? f.sx0[pol] : 0;
        const int pitch = compact ? kcount : Nx, o0 = compact ? kbeg : 0;
        float2* out = q.plane + ((size_t)unit * H + r0) * pitch;
        for (int e = tid; e < RR * kcount; e += 256) {
            const int rr = e / kcount, k = kbeg + (e - rr * kcount);
            const float2 zk = A[rr * RN + (k & (RN - 1))];
            const float2 zc = cconj(A[rr * RN + ((RN - k) & (RN - 1))]);
            const float2 even = cscale(cadd(zk, zc), 0.5f);
            const float2 d = csub(zk, zc);
            const float2 odd = make_float2(0.5f * d.y, -0.5f * d.x);
            const float2 wk = __ldg(&f.twiddle[k << (TW_LOG - 9)]);
            out[(size_t)rr * pitch + (k - o0)] = cadd(even, cmul(wk, odd));
        }
    }
}

}  // namespace


namespace {

constexpr int WC = 8;            // window columns per block
constexpr int WT = 512;          // threads per block
constexpr int WEX = 65;          // padded stride of the exchange and of Z

// One block: WC columns c0 .. c0 + 7 of one (frame, polarisation), from the
// compact row output ([unit][H][w]).  H = 64 Q rows, Q <= 8, so the
// WC Q <= 64 decimated transforms take one pass of 64 x 8 threads: thread
// (a2, s) with s = tid mod 64 the transform (column s / Q, sequence s mod Q)
// and a2 = tid / 64 its slot.
__global__ void __launch_bounds__(WT) k_plane_window64(DhFourierParams q) {
    extern __shared__ float2 sw[];
    const DhFwdParams& f = q.f;
    const int H = 1 << f.logH, Q = H >> 6;
    const int P = f.polCount, w = f.w;
    const int cgroups = w / WC;
    const int unit = blockIdx.x / cgroups, c0 = (blockIdx.x % cgroups) * WC;
    const int pol = unit % P, frame = unit / P;
    const int HS = H + 8;                       // padded column stride of S
    float2* S = sw;                             // [WC][HS]: the columns, then Z [s][WEX]
    float2* Ex = sw + WC * HS;                  // [8 k1][8 a2][WEX]
    const int tid = threadIdx.x;
    const float2* pl = q.plane + (size_t)unit * H * w + c0;
    // columns in: 8 consecutive complex values (64 bytes) of each row
    for (int e = tid; e < H * (WC / 2); e += WT) {
        const int n = e / (WC / 2), cc = 2 * (e - n * (WC / 2));
        const float4 u = *reinterpret_cast<const float4*>(pl + (size_t)n * w + cc);
        S[cc * HS + n] = make_float2(u.x, u.y);
        S[(cc + 1) * HS + n] = make_float2(u.z, u.w);
    }
    __syncthreads();
    // Z_b[k] = 64-point DFT of x_b[a] = S[c][Q a + b], a = 8 a1 + a2, k = k1 + 8 k2
    const int NS = WC * Q;
    const int s = tid & 63, a2 = tid >> 6;
    const bool act = s < NS;
    const int c = act ? s / Q : 0, b = act ? s - (s / Q) * Q : 0;
    float2 v[8];
#pragma unroll
    for (int a1 = 0; a1 < 8; a1++) v[a1] = act ? S[c * HS + Q * (8 * a1 + a2) + b] : make_float2(0.f, 0.f);
    dft8(v);
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) {
        float2 y = v[k1];
        if (k1 && a2) y = cmul(y, __ldg(&f.twiddle[(a2 * k1) << (TW_LOG - 6)]));   // exp(-2 pi i a2 k1 / 64)
        Ex[(k1 * 8 + a2) * WEX + s] = y;
    }
    __syncthreads();
    // slot a2 now takes k1 = a2: the DFT over the eight a2 values
#pragma unroll
    for (int a = 0; a < 8; a++) v[a] = Ex[(a2 * 8 + a) * WEX + s];
    dft8(v);
    // every read of S is done (the first barrier): Z[s][k] takes its place
    float2* Z = S;
    if (act) {
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) Z[s * WEX + a2 + 8 * k2] = v[k2];
    }
    __syncthreads();
    // the kept rows j: X[row_j] = sum_b exp(-2 pi i row_j b / H) Z_b[row_j mod 64],
    // row_j = (j + SY + H/2) mod H; then the batch calibration and the window factors
    float2 bc = make_float2(1.0f, 0.0f);
    if (f.batchCal && f.batchCalCount > 0)
        bc = f.batchCal[pol * f.batchCalCount + ((f.frameOffset + frame) % f.batchCalCount)];
    {
        const int j = tid & 63, cc = tid >> 6;   // 64 rows x 8 columns
        const int row = ((j + f.sy[pol] + H / 2) % H + H) % H;
        const int m = row & 63;
        const float2* tc = f.tabCol + ((size_t)pol * 64 + j) * Q;
        float2 Y = Z[(cc * Q) * WEX + m];
        for (int bb = 1; bb < Q; bb++) Y = cadd(Y, cmul(Z[(cc * Q + bb) * WEX + m], __ldg(&tc[bb])));
        Y = cmul(Y, bc);
        f.window[((size_t)unit * 64 + j) * w + c0 + cc] =
            cmul(Y, __ldg(&f.tabAdj[((size_t)pol * 64 + j) * w + c0 + cc]));
    }
}

}  // namespace

// Whether the column kernel applies: 64 x 64 Fourier windows (w a multiple of
// 8 up to 64, h = 64) in FFT windows of 128 to 512 rows, the tables present.
bool dh_plane_window64_fits(const DhFourierParams& q) {
    const DhFwdParams& f = q.f;
    const int H = 1 << f.logH;
    return f.h == 64 && f.w > 0 && f.w <= 64 && f.w % WC == 0 && H >= 128 && H <= 512 && f.tabCol && f.tabAdj &&
           f.twiddle && q.plane;
}

// Row transforms of 512-pixel FFT windows: the plane's kept columns
// (q.windowCols) or all 257, in the plane's layout, or compact
// ([unit][H][w], the kept columns only) for k_plane_window64.
// cudaErrorNotSupported where the shape or the alignment of the frame rows
// (16-byte loads) does not fit.
cudaError_t dh_launch_plane_rows512(const DhFourierParams& q, int compact, cudaStream_t s) {
    const DhFwdParams& f = q.f;
    if (f.logW != 9 || f.logH < 4 || !f.twiddle || !q.plane) return cudaErrorNotSupported;
    if (compact && !q.windowCols) return cudaErrorNotSupported;
    const size_t es = f.inputU16 ? 2 : 4;
    if ((reinterpret_cast<uintptr_t>(f.frames) & 15) || ((size_t)f.frameWidth * es) % 16 ||
        ((size_t)f.frameStride * es) % 16)
        return cudaErrorNotSupported;
    for (int p = 0; p < f.polCount; p++) {
        if (f.cx[p] < 0 || f.cy[p] < 0 || ((size_t)f.cx[p] * es) % 16) return cudaErrorNotSupported;
        if (q.windowCols && (f.sx0[p] < 0 || f.sx0[p] + f.w > RN + 1)) return cudaErrorNotSupported;
    }
    const int units = f.frameCount * f.polCount;
    if (units <= 0) return cudaSuccess;
    const size_t smem = sizeof(float2) * (size_t)RR * RN;
    const unsigned blocks = (unsigned)((units * ((1 << f.logH) / RR) + NG - 1) / NG);
    if (f.inputU16) {
        k_plane_rows512<true><<<blocks, 256, smem, s>>>(q, compact);
    } else {
        k_plane_rows512<false><<<blocks, 256, smem, s>>>(q, compact);
    }
    return cudaGetLastError();
}

// The 64-row Fourier windows with their factors from the compact row output
// of dh_launch_plane_rows512.
cudaError_t dh_launch_plane_window64(const DhFourierParams& q, cudaStream_t s) {
    const DhFwdParams& f = q.f;
    if (!dh_plane_window64_fits(q)) return cudaErrorNotSupported;
    if (reinterpret_cast<uintptr_t>(q.plane) & 15) return cudaErrorNotSupported;
    const int units = f.frameCount * f.polCount;
    if (units <= 0) return cudaSuccess;
    const int H = 1 << f.logH;
    const size_t smem = sizeof(float2) * ((size_t)WC * (H + 8) + (size_t)64 * WEX);
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_plane_window64), (int)smem);
    if (e != cudaSuccess) return e;
    k_plane_window64<<<(unsigned)(units * (f.w / WC)), WT, smem, s>>>(q);
    return cudaGetLastError();
}
