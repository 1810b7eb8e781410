// Inverse stage for low-resolution fields (IFFTResolutionMode 1, square
// IFFT windows of 16 or 32 pixels): window IFFT -> field statistics ->
// reference wave, -conj, int16 rounding -> separable HG overlap, with the
// same results as k_inverse (and as the reference's FFTW c2c backward
// digHolo.cpp:8734, digHoloFieldAnalysis digHolo.cpp:2354, applyTilt16
// digHolo.cpp:2701-2837 and overlapFieldSeparable16 digHolo.cpp:2149-2341).
//
// One group of L lanes per (frame, polarisation) unit (two units per warp
// for L = 16), no block-wide barriers: lane l transforms row l of the
// window in registers, the rows are transposed through a per-unit shared
// tile, lane l transforms column l and then owns the L pixels of field
// column x = l.  Statistics are reduced with shuffles inside the group; the
// overlap first contracts each column with Hy (U[x][n] = sum_y Hy[n][y] V[y][x]),
// then the group contracts U with Hx for its modes.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"
#include "dh_twiddle128.h"

using namespace dh;

namespace {

template <int LOG>
__host__ __device__ constexpr int brevL(int i) {
    int r = 0;
    for (int b = 0; b < LOG; b++) r |= ((i >> b) & 1) << (LOG - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2L(int n) { return n <= 1 ? 0 : 1 + ilog2L(n / 2); }

// In-place radix-2 DIF inverse FFT (exp(+2 pi i / N), unnormalised) of N <= 64
// values in registers: natural-order input, bit-reversed output.
template <int N>
__device__ __forceinline__ void ifftDIF(float2 (&v)[N]) {
#pragma unroll
    for (int m = N / 2; m >= 1; m >>= 1) {
#pragma unroll
        for (int blk = 0; blk < N; blk += 2 * m) {
#pragma unroll
            for (int j = 0; j < m; j++) {
                const float2 a = v[blk + j];
                const float2 b = v[blk + j + m];
                v[blk + j] = cadd(a, b);
                const float2 d = csub(a, b);
                if (j == 0) {
                    v[blk + j + m] = d;
                } else if (2 * j == m) {
                    v[blk + j + m] = make_float2(-d.y, d.x);   // multiply by +i
                } else {
                    const float2 t = tw128(j * (128 / (2 * m)));
                    v[blk + j + m] = cmul(d, make_float2(t.x, -t.y));
                }
            }
        }
    }
}

struct Stat {
    float maxI;
    int maxIdx;
    float P, cx, cy, cyw, e4;
};

// Reduction over the L lanes of one unit (gmask: those lanes).
template <int L>
__device__ __forceinline__ void groupReduce(Stat& s, unsigned gmask) {
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) {
        const float mI = __shfl_xor_sync(gmask, s.maxI, off);
        const int mIdx = __shfl_xor_sync(gmask, s.maxIdx, off);
        if (mI > s.maxI || (mI == s.maxI && mIdx > s.maxIdx)) { s.maxI = mI; s.maxIdx = mIdx; }
        s.P += __shfl_xor_sync(gmask, s.P, off);
        s.cx += __shfl_xor_sync(gmask, s.cx, off);
        s.cy += __shfl_xor_sync(gmask, s.cy, off);
        s.cyw += __shfl_xor_sync(gmask, s.cyw, off);
        s.e4 += __shfl_xor_sync(gmask, s.e4, off);
    }
}

constexpr int LO_WARPS = 2;

}  // namespace

// L: field side (h = w = L).  blockDim.x = 32 * LO_WARPS.
template <int L>
__global__ void __launch_bounds__(32 * LO_WARPS) k_inverse_lo(DhInvParams p) {
    constexpr int LOG = ilog2L(L);
    constexpr int UPW = 32 / L;                 // units per warp
    constexpr int UPB = UPW * LO_WARPS;         // units per block
    constexpr int npix = L * L;
    extern __shared__ float smf[];
    const int P = p.polCount;
    const int G = p.maxMG;
    const int M = p.modeCount;
    const int ULD = (G + 1) | 1;                // odd U row stride: conflict-free 8-byte stores
    const int tileC = L * (ULD > L + 1 ? ULD : L + 1);   // complex elements per unit tile

    // block tables: hx, hy [pol][G][L + 1] float (padded rows); yAxis [L];
    // mode -> (m, n)
    constexpr int HLD = L + 1;
    float* hx = smf;
    float* hy = hx + P * G * HLD;
    float* yax = hy + P * G * HLD;
    float* hsc = yax + L;                                   // [x, y][P][G] mode scales
    int* refs = reinterpret_cast<int*>(hsc + 2 * P * G);    // [P][Xr Xi Yr Yi][L] 14-bit wave
    int* modeMN = refs + P * 4 * L;
    float2* tiles = reinterpret_cast<float2*>(modeMN + ((M + 1) & ~1));
    // 8 mode values per 16-byte load: the tables arrive in about one round of loads
    for (int e = threadIdx.x; e < P * G * L / 8; e += blockDim.x) {
        const int row = (8 * e) / L, x0 = 8 * e - row * L;
        const uint4 ax = __ldg(reinterpret_cast<const uint4*>(p.hgX) + e);
        const uint4 ay = __ldg(reinterpret_cast<const uint4*>(p.hgY) + e);
        const unsigned wx[4] = {ax.x, ax.y, ax.z, ax.w}, wy[4] = {ay.x, ay.y, ay.z, ay.w};
#pragma unroll
        for (int t = 0; t < 8; t++) {
            hx[row * HLD + x0 + t] = (float)(short)((wx[t >> 1] >> (16 * (t & 1))) & 0xFFFFu);
            hy[row * HLD + x0 + t] = (float)(short)((wy[t >> 1] >> (16 * (t & 1))) & 0xFFFFu);
        }
    }
    for (int e = threadIdx.x; e < L; e += blockDim.x) yax[e] = p.yAxis[e];
    // the wave and the scales in shared memory: no global load waits behind
    // the field and coefficient stores
    for (int e = threadIdx.x; e < P * 4 * L; e += blockDim.x) refs[e] = p.refWave[e];
    for (int e = threadIdx.x; e < P * G; e += blockDim.x) {
        hsc[e] = p.hgScaleX[e];
        hsc[P * G + e] = p.hgScaleY[e];
    }
    for (int mode = threadIdx.x; mode < M; mode += blockDim.x) {
        // mode -> (m, n): group g, n = mode - g(g+1)/2, m = g - n (digHolo.cpp:1245-1265)
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2;
        modeMN[mode] = ((g - n) << 16) | n;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int ln = lane & (L - 1);
    const int slot = (threadIdx.x >> 5) * UPW + lane / L;   // unit slot within the block
    const int unit = blockIdx.x * UPB + slot;
    const int units = p.frameCount * P;
    if (unit >= units) return;   // whole groups leave together; no block barrier follows
    const unsigned gmask = (UPW == 1) ? 0xffffffffu : (0xffffu << (lane & 16));
    const int pol = unit % P, frame = unit / P;
    float2* tile = tiles + (size_t)slot * tileC;

    // 1. row ln of the window, inverse FFT over kx, transpose through the tile
    float2 v[L];
    {
        const float4* src = reinterpret_cast<const float4*>(p.window + ((size_t)unit * L + ln) * L);
#pragma unroll
        for (int q = 0; q < L / 2; q++) {
            const float4 t = __ldg(src + q);
            v[2 * q] = make_float2(t.x, t.y);
            v[2 * q + 1] = make_float2(t.z, t.w);
        }
    }
    ifftDIF<L>(v);
#pragma unroll
    for (int i = 0; i < L; i++) tile[ln * (L + 1) + brevL<LOG>(i)] = v[i];
    __syncwarp(gmask);
#pragma unroll
    for (int j = 0; j < L; j++) v[j] = tile[j * (L + 1) + ln];
    __syncwarp(gmask);
    // 2. column x = ln over ky: v[i] = F[y = brev(i)][x = ln]
    ifftDIF<L>(v);

    // 3. statistics over the untilted field (digHolo.cpp:8866-8870)
    const float inv = (float)(1.0 / ((double)L * (double)L));
    const float yShift = fabsf((yax[1] - yax[0]) * (float)L);
    const float xv = p.xAxis[ln];
    Stat st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < L; i++) {
        const int y = brevL<LOG>(i);
        const float2 a = v[i];
        const float I0 = fmaf(a.x, a.x, a.y * a.y);
        const float I = I0 * inv;
        const int idx = 2 * y * L + ln;
        if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
        const float yv = yax[y];
        st.P += I;
        st.cx = fmaf(xv, I, st.cx);
        st.cy = fmaf(yv, I, st.cy);
        st.cyw = fmaf(yv + (yv < 0.f ? yShift : 0.f), I, st.cyw);
        st.e4 = fmaf(I, I, st.e4);
    }
    groupReduce<L>(st, gmask);
    const float maxAbs = sqrtf(st.maxI);
    const float scale = (float)(32767.0 / (double)maxAbs);
    if (ln == 0) {
        const int S = p.statsStride;
        float* s = p.stats;
        const int col = pol * S + frame;
        const int per = P * S;
        s[0 * per + col] = st.P;
        s[1 * per + col] = st.cx / st.P;
        s[2 * per + col] = st.cy / st.P;
        s[3 * per + col] = scale;
        s[4 * per + col] = __int_as_float(st.maxIdx);
        s[5 * per + col] = p.dA * (st.P * st.P / st.e4);
        s[6 * per + col] = st.cyw / st.P;
    }

    // 4. reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833)
    const int* ref = refs + (size_t)pol * 4 * L;
    const int xr = ref[ln], xi = ref[L + ln];
    const float K = (float)(1.0 / (16383.0 * 16383.0));
    const size_t fieldOff = (size_t)unit * npix;
    float2 V[L];
#pragma unroll
    for (int i = 0; i < L; i++) {
        const int y = brevL<LOG>(i);
        const int yr = ref[2 * L + y], yi = ref[3 * L + y];
        const float adjR = (float)(yr * xr - yi * xi) * K;
        const float adjI = (float)(yr * xi + yi * xr) * K;
        const float2 a = v[i];
        const float vr = __fsub_rn(__fmul_rn(a.y, adjI), __fmul_rn(a.x, adjR));
        const float vi = __fadd_rn(__fmul_rn(a.x, adjI), __fmul_rn(a.y, adjR));
        const size_t o = fieldOff + (size_t)y * L + ln;
        if (p.field32) {
            const float* rf = p.refWaveF + (size_t)pol * 4 * L;
            const float2 rx = make_float2(rf[ln], rf[L + ln]);
            const float2 ry = make_float2(rf[2 * L + y], rf[3 * L + y]);
            const float2 w = cmul(a, cmul(ry, rx));
            p.field32[o] = make_float2(-w.x, w.y);
        }
        const short sr = roundSat16(scale * vr);
        const short si = roundSat16(scale * vi);
        p.fieldR[o] = sr;
        p.fieldI[o] = si;
        V[i] = make_float2((float)sr, (float)si);
    }
    if (G <= 0 || !p.coefs) return;

    // 5. overlap on the int16 field (digHolo.cpp:2149-2341), contracted over y
    //    first: U[x][n] = sum_y Hy[n][y] V[y][x]; c_mn = sum_x Hx[m][x] U[x][n]
    const float* hyp = hy + (size_t)pol * G * HLD;
    const float* hxp = hx + (size_t)pol * G * HLD;
    float2* U = tile;   // [x][ULD], the transposed tile is dead
    for (int n = 0; n < G; n++) {
        const float* hn = hyp + n * HLD;
        float ur = 0.f, ui = 0.f;
#pragma unroll
        for (int i = 0; i < L; i++) {
            const float hv = hn[brevL<LOG>(i)];
            ur = fmaf(hv, V[i].x, ur);
            ui = fmaf(hv, V[i].y, ui);
        }
        U[ln * ULD + n] = make_float2(ur, ui);
    }
    __syncwarp(gmask);
    const float fieldScale = 1.0f / scale;
    const float* sxp = hsc + pol * G;
    const float* syp = hsc + P * G + pol * G;
    float2* cout = p.coefs + (size_t)frame * P * M + (size_t)pol * M;
    for (int mode = ln; mode < M; mode += L) {
        const int mn = modeMN[mode];
        const int m = mn >> 16, n = mn & 0xFFFF;
        const float* hm = hxp + m * HLD;
        float cr = 0.f, ci = 0.f;
#pragma unroll
        for (int x = 0; x < L; x++) {
            const float2 u = U[x * ULD + n];
            cr = fmaf(hm[x], u.x, cr);
            ci = fmaf(hm[x], u.y, ci);
        }
        const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
        cout[mode] = make_float2(cr * ms, ci * ms);
    }
}

// Returns cudaErrorNotSupported for shapes this kernel does not cover.
cudaError_t dh_launch_inverse_lo(const DhInvParams& p, cudaStream_t s) {
    if (!p.lowres || p.logw != p.logh || (p.logw != 4 && p.logw != 5)) return cudaErrorNotSupported;
    if (p.w != (1 << p.logw) || p.h != (1 << p.logh)) return cudaErrorNotSupported;   // power-of-two windows only
    // the table loads read 16-byte chunks of the int16 modes
    if (p.maxMG > 0 && ((reinterpret_cast<uintptr_t>(p.hgX) | reinterpret_cast<uintptr_t>(p.hgY)) & 15))
        return cudaErrorNotSupported;
    const int L = 1 << p.logw;
    const int units = p.frameCount * p.polCount;
    if (units <= 0) return cudaSuccess;
    const int G = p.maxMG > 0 ? p.maxMG : 0;
    const int M = p.maxMG > 0 ? p.modeCount : 0;
    const int ULD = (G + 1) | 1;
    const int UPB = (32 / L) * LO_WARPS;
    const size_t smem = sizeof(float) * ((size_t)2 * p.polCount * G * (L + 1) + L + 2 * (size_t)p.polCount * G) +
                        sizeof(int) * ((size_t)p.polCount * 4 * L + (size_t)((M + 1) & ~1)) +
                        sizeof(float2) * (size_t)UPB * L * (ULD > L + 1 ? ULD : L + 1);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    DhInvParams q = p;
    q.maxMG = G;
    q.modeCount = M;
    const unsigned blocks = (unsigned)((units + UPB - 1) / UPB);
    cudaError_t e;
    if (L == 16) {
        e = setSmemOnce(reinterpret_cast<const void*>(k_inverse_lo<16>), (int)smem);
        if (e != cudaSuccess) return e;
        k_inverse_lo<16><<<blocks, 32 * LO_WARPS, smem, s>>>(q);
    } else {
        e = setSmemOnce(reinterpret_cast<const void*>(k_inverse_lo<32>), (int)smem);
        if (e != cudaSuccess) return e;
        k_inverse_lo<32><<<blocks, 32 * LO_WARPS, smem, s>>>(q);
    }
    return cudaGetLastError();
}
