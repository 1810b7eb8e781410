// Inverse stage for low-resolution fields (IFFTResolutionMode 1, square
// IFFT windows of 16 or 32 pixels): window IFFT -> field statistics ->
// reference wave, -conj, int16 rounding -> separable HG overlap, with the
// same results as k_inverse (and as the reference's FFTW c2c backward
// digHolo.cpp:8734, digHoloFieldAnalysis digHolo.cpp:2354, applyTilt16
// digHolo.cpp:2701-2837 and overlapFieldSeparable16 digHolo.cpp:2149-2341).
//
// k_inverse_lo<32>: one warp per (frame, polarisation) unit, no block-wide
// barriers: lane l transforms row l of the window in registers, the rows are
// transposed through a per-unit shared tile, lane l transforms column l and
// then owns the L pixels of field column x = l.  Statistics are reduced with
// shuffles; the overlap first contracts each column with Hy
// (U[x][n] = sum_y Hy[n][y] V[y][x]), then the warp contracts U with Hx for
// its modes.
// k_inverse_lo16q (16-pixel fields): the same steps with 64 threads per
// unit, a quad of lanes per row and column transform (see there).
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

namespace {

constexpr int Q_UNITS = 4;                  // units per block of the 16-pixel kernel
constexpr int Q_THREADS = 64 * Q_UNITS;     // 64 threads per unit
constexpr int Q_TLD = 20;                   // tile row stride (complex): conflict-free quad accesses

// w^k, w = exp(+2 pi i / 16), from the same float table as the radix-2 passes
__device__ __forceinline__ float2 w16(int k) {
    const float2 t = tw128(8 * k);
    return make_float2(t.x, -t.y);
}

// y[b] = sum_a x[a] i^(ab): the 4-point inverse DFT
__device__ __forceinline__ void idft4(float2& x0, float2& x1, float2& x2, float2& x3) {
    const float2 s02 = cadd(x0, x2), d02 = csub(x0, x2);
    const float2 s13 = cadd(x1, x3), d13 = csub(x1, x3);
    const float2 id13 = make_float2(-d13.y, d13.x);
    x0 = cadd(s02, s13);
    x2 = csub(s02, s13);
    x1 = cadd(d02, id13);
    x3 = csub(d02, id13);
}

// Barrier of one unit's 64 threads (named barrier 1 + slot): after the
// block-wide barrier that publishes the tables, the units of a block share
// nothing, so each waits only for its own two warps.
__device__ __forceinline__ void unitBar(int slot) { asm volatile("bar.sync %0, 64;" ::"r"(1 + slot) : "memory"); }

__device__ __forceinline__ float2 shflXor2(float2 v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// 16-point inverse DFT (exp(+2 pi i nk / 16), unnormalised) of one line held
// by the 4 lanes of a quad: lane q holds u[q + 4a] in x[a] on entry and
// U[q + 4c] in x[c] on exit.  With n = q + 4a and k = b + 4c,
// U[b + 4c] = sum_q i^(qc) w^(qb) sum_a u[q + 4a] i^(ab): a 4-point DFT in
// each lane, the twiddles w^(qb), a 4 x 4 transpose across the quad (two
// exchange rounds of shuffles) and a second 4-point DFT.
__device__ __forceinline__ void ifft16Quad(float2 (&x)[4], int q, const float2 (&tw)[4]) {
    idft4(x[0], x[1], x[2], x[3]);
    x[1] = cmul(x[1], tw[1]);
    x[2] = cmul(x[2], tw[2]);
    x[3] = cmul(x[3], tw[3]);
    // round A (lanes q, q ^ 2): keep the two b with bit 1 of b equal to bit 1 of q
    const bool hi = (q & 2) != 0;
    const float2 r0 = shflXor2(hi ? x[0] : x[2], 2);
    const float2 r1 = shflXor2(hi ? x[1] : x[3], 2);
    const float2 a0 = hi ? x[2] : x[0], a1 = hi ? x[3] : x[1];   // own, b = (q & 2) + 0 / 1
    // round B (lanes q, q ^ 1): keep b = q
    const bool lo = (q & 1) != 0;
    const float2 s0 = shflXor2(lo ? a0 : a1, 1);   // source q ^ 1
    const float2 s1 = shflXor2(lo ? r0 : r1, 1);   // source q ^ 3
    const float2 k0 = lo ? a1 : a0;                // source q
    const float2 k1 = lo ? r1 : r0;                // source q ^ 2
    // order by source lane: v[q ^ d] for d = 0, 1, 2, 3
    float2 v0, v1, v2, v3;
    switch (q) {
        case 0: v0 = k0; v1 = s0; v2 = k1; v3 = s1; break;
        case 1: v0 = s0; v1 = k0; v2 = s1; v3 = k1; break;
        case 2: v0 = k1; v1 = s1; v2 = k0; v3 = s0; break;
        default: v0 = s1; v1 = k1; v2 = s0; v3 = k0; break;
    }
    idft4(v0, v1, v2, v3);
    x[0] = v0; x[1] = v1; x[2] = v2; x[3] = v3;
}

}  // namespace

// 16 x 16 low-resolution fields with 64 threads per (frame, polarisation)
// unit, Q_UNITS units per block: each quad of lanes transforms one row and
// then one column (ifft16Quad), so a thread ends with the four pixels
// (x = t / 4, y = t % 4 + 4c); statistics reduce over the unit's two warps,
// and the overlap spreads its U[x][n] and mode sums over all 64 threads.
// The same steps and roundings as k_inverse_lo<16>, four times the threads:
// 2048 units fill ~28 warps per SM instead of 7.
__global__ void __launch_bounds__(Q_THREADS) k_inverse_lo16q(DhInvParams p) {
    constexpr int L = 16;
    constexpr int npix = L * L;
    extern __shared__ float smf[];
    const int P = p.polCount;
    const int G = p.maxMG;
    const int M = p.modeCount;
    const int ULD = (G + 1) | 1;
    constexpr int HLD = L + 1;
    const int tid = threadIdx.x;
    const int slot = tid >> 6, t = tid & 63;
    const int q = t & 3, line = t >> 2;
    const int unit = blockIdx.x * Q_UNITS + slot;
    const int units = p.frameCount * P;
    const bool active = unit < units;
    const int pol = active ? unit % P : 0, frame = active ? unit / P : 0;

    // 0. this thread's window values first (their loads overlap the tables):
    //    row `line`, columns q + 4a
    float2 x[4];
    if (active) {
        const float2* src = p.window + ((size_t)unit * L + line) * L + q;
#pragma unroll
        for (int a = 0; a < 4; a++) x[a] = __ldg(src + 4 * a);
    } else {
#pragma unroll
        for (int a = 0; a < 4; a++) x[a] = make_float2(0.f, 0.f);
    }

    float* hx = smf;
    float* hy = hx + P * G * HLD;
    float* yax = hy + P * G * HLD;
    float* hsc = yax + L;
    int* refs = reinterpret_cast<int*>(hsc + 2 * P * G);
    int* modeMN = refs + P * 4 * L;
    float* red = reinterpret_cast<float*>(modeMN + ((M + 1) & ~1));      // [unit][warp][8]
    float2* tiles = reinterpret_cast<float2*>(red + Q_UNITS * 2 * 8);   // 8-byte aligned: offsets are even
    const int tileC = L * Q_TLD + L * ULD;
    float2* T = tiles + (size_t)slot * tileC;    // [16][Q_TLD]: rows, then the int16 field
    float2* U = T + L * Q_TLD;                   // [16][ULD]
    for (int e = tid; e < P * G * L / 8; e += Q_THREADS) {
        const int row = (8 * e) / L, x0 = 8 * e - row * L;
        const uint4 ax = __ldg(reinterpret_cast<const uint4*>(p.hgX) + e);
        const uint4 ay = __ldg(reinterpret_cast<const uint4*>(p.hgY) + e);
        const unsigned wx[4] = {ax.x, ax.y, ax.z, ax.w}, wy[4] = {ay.x, ay.y, ay.z, ay.w};
#pragma unroll
        for (int k = 0; k < 8; k++) {
            hx[row * HLD + x0 + k] = (float)(short)((wx[k >> 1] >> (16 * (k & 1))) & 0xFFFFu);
            hy[row * HLD + x0 + k] = (float)(short)((wy[k >> 1] >> (16 * (k & 1))) & 0xFFFFu);
        }
    }
    for (int e = tid; e < L; e += Q_THREADS) yax[e] = p.yAxis[e];
    for (int e = tid; e < P * 4 * L; e += Q_THREADS) refs[e] = p.refWave[e];
    for (int e = tid; e < P * G; e += Q_THREADS) {
        hsc[e] = p.hgScaleX[e];
        hsc[P * G + e] = p.hgScaleY[e];
    }
    for (int mode = tid; mode < M; mode += Q_THREADS) {
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2;
        modeMN[mode] = ((g - n) << 16) | n;
    }
    float2 tw[4];
    tw[0] = make_float2(1.f, 0.f);
    tw[1] = q == 0 ? w16(0) : (q == 1 ? w16(1) : (q == 2 ? w16(2) : w16(3)));
    tw[2] = q == 0 ? w16(0) : (q == 1 ? w16(2) : (q == 2 ? w16(4) : w16(6)));
    tw[3] = q == 0 ? w16(0) : (q == 1 ? w16(3) : (q == 2 ? w16(6) : w16(9)));

    // 1. row `line` over kx: R[ky = line][x = q + 4c]
    ifft16Quad(x, q, tw);
#pragma unroll
    for (int c = 0; c < 4; c++) T[line * Q_TLD + q + 4 * c] = x[c];
    __syncthreads();
    // 2. column x = line over ky: F[y = q + 4c][x = line]
#pragma unroll
    for (int a = 0; a < 4; a++) x[a] = T[(q + 4 * a) * Q_TLD + line];
    ifft16Quad(x, q, tw);

    // 3. statistics over the untilted field (digHolo.cpp:8866-8870)
    const float inv = (float)(1.0 / ((double)L * (double)L));
    const float yShift = fabsf((yax[1] - yax[0]) * (float)L);
    const int xpix = line;
    const float xv = p.xAxis[xpix];
    Stat st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int y = q + 4 * c;
        const float2 a = x[c];
        const float I0 = fmaf(a.x, a.x, a.y * a.y);
        const float I = I0 * inv;
        const int idx = 2 * y * L + xpix;
        if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
        const float yv = yax[y];
        st.P += I;
        st.cx = fmaf(xv, I, st.cx);
        st.cy = fmaf(yv, I, st.cy);
        st.cyw = fmaf(yv + (yv < 0.f ? yShift : 0.f), I, st.cyw);
        st.e4 = fmaf(I, I, st.e4);
    }
    groupReduce<32>(st, 0xffffffffu);
    float* rw = red + (slot * 2 + (t >> 5)) * 8;
    if ((t & 31) == 0) {
        rw[0] = st.maxI; rw[1] = __int_as_float(st.maxIdx);
        rw[2] = st.P; rw[3] = st.cx; rw[4] = st.cy; rw[5] = st.cyw; rw[6] = st.e4;
    }
    unitBar(slot);
    {
        const float* r0 = red + slot * 16;
        const float* r1 = r0 + 8;
        const float m0 = r0[0], m1 = r1[0];
        const int i0 = __float_as_int(r0[1]), i1 = __float_as_int(r1[1]);
        const bool take1 = m1 > m0 || (m1 == m0 && i1 > i0);
        st.maxI = take1 ? m1 : m0;
        st.maxIdx = take1 ? i1 : i0;
        st.P = r0[2] + r1[2];
        st.cx = r0[3] + r1[3];
        st.cy = r0[4] + r1[4];
        st.cyw = r0[5] + r1[5];
        st.e4 = r0[6] + r1[6];
    }
    const float maxAbs = sqrtf(st.maxI);
    const float scale = (float)(32767.0 / (double)maxAbs);
    if (active && t == 0) {
        const int S = p.statsStride;
        float* sp = p.stats;
        const int col = pol * S + frame;
        const int per = P * S;
        sp[0 * per + col] = st.P;
        sp[1 * per + col] = st.cx / st.P;
        sp[2 * per + col] = st.cy / st.P;
        sp[3 * per + col] = scale;
        sp[4 * per + col] = __int_as_float(st.maxIdx);
        sp[5 * per + col] = p.dA * (st.P * st.P / st.e4);
        sp[6 * per + col] = st.cyw / st.P;
    }

    // 4. reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833);
    //    the int16 field into T (its rows were read before the barrier above)
    const int* ref = refs + (size_t)pol * 4 * L;
    const int xr = ref[xpix], xi = ref[L + xpix];
    const float K = (float)(1.0 / (16383.0 * 16383.0));
    const size_t fieldOff = (size_t)unit * npix;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int y = q + 4 * c;
        const int yr = ref[2 * L + y], yi = ref[3 * L + y];
        const float adjR = (float)(yr * xr - yi * xi) * K;
        const float adjI = (float)(yr * xi + yi * xr) * K;
        const float2 a = x[c];
        const float vr = __fsub_rn(__fmul_rn(a.y, adjI), __fmul_rn(a.x, adjR));
        const float vi = __fadd_rn(__fmul_rn(a.x, adjI), __fmul_rn(a.y, adjR));
        const short sr = roundSat16(scale * vr);
        const short si = roundSat16(scale * vi);
        if (active) {
            const size_t o = fieldOff + (size_t)y * L + xpix;
            if (p.field32) {
                const float* rf = p.refWaveF + (size_t)pol * 4 * L;
                const float2 rx = make_float2(rf[xpix], rf[L + xpix]);
                const float2 ry = make_float2(rf[2 * L + y], rf[3 * L + y]);
                const float2 w = cmul(a, cmul(ry, rx));
                p.field32[o] = make_float2(-w.x, w.y);
            }
            p.fieldR[o] = sr;
            p.fieldI[o] = si;
        }
        T[y * Q_TLD + xpix] = make_float2((float)sr, (float)si);
    }
    if (G <= 0 || !p.coefs) return;   // uniform over the block: no barrier is skipped by part of it
    unitBar(slot);

    // 5. overlap on the int16 field (digHolo.cpp:2149-2341):
    //    U[x][n] = sum_y Hy[n][y] V[y][x], then c_mn = sum_x Hx[m][x] U[x][n]
    const float* hyp = hy + (size_t)pol * G * HLD;
    const float* hxp = hx + (size_t)pol * G * HLD;
    {
        const int xc = t & 15;
        float2 V[L];
#pragma unroll
        for (int y = 0; y < L; y++) V[y] = T[y * Q_TLD + xc];
        for (int n = t >> 4; n < G; n += 4) {
            const float* hn = hyp + n * HLD;
            float ur = 0.f, ui = 0.f;
#pragma unroll
            for (int y = 0; y < L; y++) {
                ur = fmaf(hn[y], V[y].x, ur);
                ui = fmaf(hn[y], V[y].y, ui);
            }
            U[xc * ULD + n] = make_float2(ur, ui);
        }
    }
    unitBar(slot);
    if (!active) return;
    const float fieldScale = 1.0f / scale;
    const float* sxp = hsc + pol * G;
    const float* syp = hsc + P * G + pol * G;
    float2* cout = p.coefs + (size_t)frame * P * M + (size_t)pol * M;
    for (int mode = t; mode < M; mode += 64) {
        const int mn = modeMN[mode];
        const int m = mn >> 16, n = mn & 0xFFFF;
        const float* hm = hxp + m * HLD;
        float cr = 0.f, ci = 0.f;
#pragma unroll
        for (int xx = 0; xx < L; xx++) {
            const float2 u = U[xx * ULD + n];
            cr = fmaf(hm[xx], u.x, cr);
            ci = fmaf(hm[xx], u.y, ci);
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
    const size_t tables = sizeof(float) * ((size_t)2 * p.polCount * G * (L + 1) + L + 2 * (size_t)p.polCount * G) +
                          sizeof(int) * ((size_t)p.polCount * 4 * L + (size_t)((M + 1) & ~1));
    DhInvParams q = p;
    q.maxMG = G;
    q.modeCount = M;
    cudaError_t e;
    if (L == 16) {
        // tables, the statistics partials, then per unit the row / field tile and U
        // (tables is a multiple of 8 bytes: every count above is even)
        const size_t smemQ = tables + sizeof(float) * Q_UNITS * 2 * 8 +
                             sizeof(float2) * (size_t)Q_UNITS * (L * Q_TLD + L * ULD);
        if (smemQ > 200 * 1024) return cudaErrorNotSupported;
        e = setSmemOnce(reinterpret_cast<const void*>(k_inverse_lo16q), (int)smemQ);
        if (e != cudaSuccess) return e;
        k_inverse_lo16q<<<(unsigned)((units + Q_UNITS - 1) / Q_UNITS), Q_THREADS, smemQ, s>>>(q);
        return cudaGetLastError();
    }
    const size_t smem = tables + sizeof(float2) * (size_t)UPB * L * (ULD > L + 1 ? ULD : L + 1);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    const unsigned blocks = (unsigned)((units + UPB - 1) / UPB);
    e = setSmemOnce(reinterpret_cast<const void*>(k_inverse_lo<32>), (int)smem);
    if (e != cudaSuccess) return e;
    k_inverse_lo<32><<<blocks, 32 * LO_WARPS, smem, s>>>(q);
    return cudaGetLastError();
}
