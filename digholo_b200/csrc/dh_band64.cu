// Inverse stage of full-resolution 512-pixel-wide fields (IFFTResolutionMode
// 0 with a 512-wide FFT window and an IFFT window of at most 64 x 64: the
// large-field workload, 2048 x 2048 frames with 512 x 512 FFT windows): the
// Fourier window placed in the H x W plane -> IFFT -> field statistics ->
// reference wave, -conj, int16 rounding -> separable HG overlap.  The same
// results as the band kernels of dh_big.cu, i.e. the reference's FFTW c2c
// backward (digHolo.cpp:8734), digHoloFieldAnalysis (digHolo.cpp:2354),
// applyTilt16 (digHolo.cpp:2701-2837) and overlapFieldSeparable16
// (digHolo.cpp:2149-2341).
//
// Transform.  E[y][x] = sum_j sum_c win[j][c] e^{2 pi i (r0 + j) y / H}
// e^{2 pi i (sx0 + c) x / W}.  With y = Ry s + u (Ry = H / 64) the column
// transform of window column c is, for every u, one 64-point inverse DFT over
// m = (r0 + j) mod 64 of win[j][c] e^{2 pi i (r0 + j) u / H}; with
// x = Rx t + v (Rx = W / 64) the row transform is, for every v, one 64-point
// inverse DFT over m = (sx0 + c) mod 64 of A[c] e^{2 pi i (sx0 + c) v / W}.
// A 64-point transform runs on four lanes, 16 points each: a 16-point DFT in
// registers, the twiddle e^{2 pi i lane s1 / 64}, and a 4-point DFT across
// the lanes by two shuffle butterflies; lane l ends with the outputs
// s1 + 16 brev2(l), s1 = 0..15.
//
// A block (512 threads) owns the band of 64 rows y = Ry s + u of one
// (frame, polarisation) field: the column transforms of its u, then the row
// transforms in passes of 128 (16 rows x 8 v).  The int16 scale depends on
// the maximum over the whole field, so a statistics pass writes one partial
// record per band and the quantising pass merges them in band order
// (identically in every block) and recomputes the band.  Quantised values
// go through a shared-memory tile to coalesced 16-byte stores of the int16
// planes and into the overlap operand.
//
// Overlap.  T[row][m] = sum_x F[row][x] Hx[m][x] of int16 F (R and I rows) and
// int16 Hx is exact in integers: with F = 256 Fh + Fl (Fh signed, Fl
// unsigned bytes) and likewise Hx, four tcgen05.mma.kind::i8 products
// (s8 x s8, s8 x u8, u8 x s8, u8 x u8; int32 accumulators in tensor memory,
// |partial| < 2^26 for K = 512) give T = 65536 hh + 256 (hl + lh) + ll.  The
// band's rows are then contracted with Hy in FP32 and a last kernel sums the
// bands and applies the mode scales.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_fft.cuh"
#include "dh_host.h"
#include "dh_params.h"
#include "dh_tc.cuh"

using namespace dh;

namespace {

constexpr int NT = 512;     // threads per block
constexpr int SLOTS = NT / 4;   // 64-point transforms per pass
constexpr int BR = 64;      // field rows per band
constexpr int WF = 512;     // field width this kernel is built for
constexpr int RX = WF / 64; // row sub-problems v
constexpr int ROWS_PP = SLOTS / RX;   // rows per row pass (16)
constexpr int NPASS = BR / ROWS_PP;   // row passes per band (4)
constexpr int GNMAX = 32;

enum { P_STATS = 0, P_QUANT = 1, P_I8 = 2 };

// cos and sin of 2 pi m / 16, m = 0..9
__device__ __constant__ float kC[10] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                                        -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f, -1.0f,
                                        -0.92387953251128674f};
__device__ __constant__ float kS[10] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f, 1.0f,
                                        0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                                        -0.38268343236508977f};

// 4-point inverse DFT in place (exp(+2 pi i / 4)), natural order.
__device__ __forceinline__ void idft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    const float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
    const float2 r = make_float2(-d13.y, d13.x);   // +i d13
    a0 = cadd(s02, s13);
    a1 = cadd(d02, r);
    a2 = csub(s02, s13);
    a3 = csub(d02, r);
}

// 16-point inverse DFT in registers, natural order in and out.
__device__ __forceinline__ void idft16(float2 (&v)[16]) {
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) idft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
#pragma unroll
    for (int k1 = 1; k1 < 4; k1++) {
#pragma unroll
        for (int n2 = 1; n2 < 4; n2++) {
            const int m = n2 * k1;
            v[4 * k1 + n2] = cmul(v[4 * k1 + n2], make_float2(kC[m], kS[m]));
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) idft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // X[k1 + 4 k2] sits at v[4 k1 + k2]: transpose the 4 x 4 index grid
    float2 t[16];
#pragma unroll
    for (int k = 0; k < 16; k++) t[k] = v[4 * (k & 3) + (k >> 2)];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = t[k];
}

// 64-point inverse DFT on the four lanes l = lane & 3 of a lane quad:
// in v[m1] = x[4 m1 + l], out v[s1] = X[s1 + 16 brev2(l)].  tw64p[k] =
// e^{2 pi i k / 64}.  All 32 lanes of the warp take part.
__device__ __forceinline__ void ifft64q(float2 (&v)[16], int l, const float2* tw64p) {
    idft16(v);
#pragma unroll
    for (int s1 = 1; s1 < 16; s1++) v[s1] = cmul(v[s1], tw64p[(l * s1) & 63]);
    // X[s2] = sum_l y_l i^{l s2}: butterflies across lane bit 1, then bit 0
    const float sA = (l & 2) ? -1.0f : 1.0f;
    const float sB = (l & 1) ? -1.0f : 1.0f;
    const bool rot = (l & 3) == 3;   // bit 0 and bit 1: times i before the second butterfly
#pragma unroll
    for (int s1 = 0; s1 < 16; s1++) {
        float2 a = v[s1];
        const float ox = __shfl_xor_sync(0xffffffffu, a.x, 2);
        const float oy = __shfl_xor_sync(0xffffffffu, a.y, 2);
        a = make_float2(fmaf(sA, a.x, ox), fmaf(sA, a.y, oy));
        if (rot) a = make_float2(-a.y, a.x);
        const float px = __shfl_xor_sync(0xffffffffu, a.x, 1);
        const float py = __shfl_xor_sync(0xffffffffu, a.y, 1);
        v[s1] = make_float2(fmaf(sB, a.x, px), fmaf(sB, a.y, py));
    }
}

__host__ __device__ constexpr int brev2(int l) { return ((l & 1) << 1) | ((l >> 1) & 1); }

// Staging-tile column of field column x (16 rows x 512 packed R | I << 16):
// bits 3-4 of x flipped by the quarter 128-column block, so that the lanes of
// a warp (8 v of one row, four quarters) store to distinct banks.
__device__ __forceinline__ int stagePhys(int x) { return x ^ (((x >> 7) & 3) << 3); }

__host__ __device__ __forceinline__ size_t alignUpD(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Shared-memory plan; the host computes the same numbers.
struct B64Smem {
    size_t planes, stage, ab, rowTw, colTw, tw, refX, refY, xAx, yAx, hy, red, bars, total;
};
__host__ __device__ inline B64Smem band64Smem(int pass, int w, int G, int GN) {
    B64Smem s;
    size_t o = 0;
    s.planes = o;
    if (pass == P_I8) o += (size_t)2 * WF * 128;          // hi, lo: [W / 128 atoms][128 rows][128 B]
    s.stage = o;
    if (pass != P_STATS) o += (size_t)ROWS_PP * WF * 4;   // packed int16 pairs; the epilogue's T after the last pass
    s.ab = o;
    size_t ab = (size_t)BR * (w + 4) * sizeof(float2);
    if (pass == P_I8 && (size_t)GN * WF * 2 > ab) ab = (size_t)GN * WF * 2;   // then Hx hi, lo
    o = alignUpD(o + ab, 1024);
    s.rowTw = o;
    o += (size_t)RX * (w + 4) * sizeof(float2);
    s.colTw = o;
    o += 64 * sizeof(float2);
    s.tw = o;
    o += 64 * sizeof(float2);
    s.refX = o;
    if (pass != P_STATS) o += (size_t)WF * 4;
    s.refY = o;
    if (pass != P_STATS) o += (size_t)BR * 8;
    s.xAx = o;
    if (pass == P_STATS) o += (size_t)WF * 4;
    s.yAx = o;
    if (pass == P_STATS) o += (size_t)BR * 4;
    s.hy = o;
    if (pass == P_I8) o += (size_t)G * BR * 4;
    s.red = o;
    o += sizeof(StatF) * (NT / 32);
    o = alignUpD(o, 8);
    s.bars = o;
    o += 2 * 8 + 8;
    s.total = o + 1024;   // room to align the base to 1024 bytes
    return s;
}

struct B64Args {
    StatF* part;                 // [unit][band] partial statistics
    float2* partCoefs;           // [unit][band][modeCount]
    const unsigned char* hx;     // [pol][hi, lo][W / 128 atoms][GN][128 B] (swizzled bytes)
};

__device__ __forceinline__ uint32_t instrDescI8s(int M, int N, bool aSigned, bool bSigned) {
    return (2u << 4) | ((aSigned ? 1u : 0u) << 7) | ((bSigned ? 1u : 0u) << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mmaI8(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tmemLoad16u(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Byte offset of the 8 bytes of K elements x0 .. x0 + 7 (x0 a multiple of 8)
// of operand row r in a K-major 128-byte-swizzled i8 operand of `rows` rows.
__device__ __forceinline__ uint32_t planeOff(int rows, int r, int x0) {
    const int atom = x0 >> 7, chunk = (x0 & 127) >> 4, half = (x0 >> 3) & 1;
    return (uint32_t)(atom * rows * 128 + r * 128 + ((chunk ^ (r & 7)) << 4) + half * 8);
}

// One block: the band of rows y = Ry s + band (s = 0..63) of one (frame,
// polarisation) field.  blockIdx.x = unit * Ry + band.
template <int PASS, int GN>
__global__ void __launch_bounds__(NT, 1) k_band64(DhInvParams p, B64Args a) {
    constexpr bool QUANT = PASS != P_STATS;
    constexpr bool I8 = PASS == P_I8;
    const int W = WF, H = 1 << p.logH, w = p.w, h = p.h;
    const int Ry = H / 64;
    const int unit = blockIdx.x / Ry, band = blockIdx.x % Ry;
    const int P = p.polCount, pol = unit % P, frame = unit / P;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int lq = tid & 3, slot = tid >> 2;
    const int G = I8 ? p.maxMG : 0, M = p.modeCount;
    const int AW = w + 4;   // padded row of Ab and rowTw

    const B64Smem L = band64Smem(PASS, w, G, GN);
    extern __shared__ float4 smf4[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smf4) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* hiPlane = base + L.planes;                          // I8: [4][128][128 B]
    unsigned char* loPlane = hiPlane + (size_t)WF * 128;
    uint32_t* stage = reinterpret_cast<uint32_t*>(base + L.stage);    // [16][512] R | I << 16
    float* Tsm = reinterpret_cast<float*>(base + L.stage);            // I8 epilogue: [128][GN + 1]
    float2* Ab = reinterpret_cast<float2*>(base + L.ab);              // [64][w + 4] column-stage output
    unsigned char* hxHi = base + L.ab;                                // I8, after the last gather: [4][GN][128 B]
    unsigned char* hxLo = hxHi + (size_t)GN * WF;
    float2* rowTw = reinterpret_cast<float2*>(base + L.rowTw);        // [RX][w + 4]
    float2* colTw = reinterpret_cast<float2*>(base + L.colTw);        // [64]
    float2* tw64p = reinterpret_cast<float2*>(base + L.tw);           // [64] e^{2 pi i k / 64}
    uint32_t* refX = reinterpret_cast<uint32_t*>(base + L.refX);      // [W] Xr | Xi << 16
    int2* refY = reinterpret_cast<int2*>(base + L.refY);              // [64] (Yr, Yi) of the band's rows
    float* xAx = reinterpret_cast<float*>(base + L.xAx);              // [W]
    float* yAx = reinterpret_cast<float*>(base + L.yAx);              // [64]
    float* hyB = reinterpret_cast<float*>(base + L.hy);               // I8: [G][64]
    StatF* red = reinterpret_cast<StatF*>(base + L.red);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + L.bars);      // I8: Hx load, MMA commit
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bars + 2);

    const int r0 = ((p.sy[pol] + H / 2) % H + H) % H;
    const int sx0 = p.sx0[pol];
    const short* ref = p.refWave + (size_t)pol * 2 * (W + H);

    // tables
    for (int e = tid; e < 64; e += NT) {
        tw64p[e] = expPos(p.twiddle, e, 64);
        colTw[e] = e < h ? expPos(p.twiddle, ((r0 + e) % H) * band, H) : make_float2(0.f, 0.f);
    }
    for (int e = tid; e < RX * w; e += NT) {
        const int v = e / w, c = e - v * w;
        rowTw[v * AW + c] = expPos(p.twiddle, ((sx0 + c) % W) * v, W);
    }
    if (QUANT) {
        for (int e = tid; e < W; e += NT)
            refX[e] = (uint32_t)(unsigned short)ref[e] | ((uint32_t)(unsigned short)ref[W + e] << 16);
        for (int e = tid; e < BR; e += NT) {
            const int y = Ry * e + band;
            refY[e] = make_int2((int)ref[2 * W + y], (int)ref[2 * W + H + y]);
        }
    } else {
        for (int e = tid; e < W; e += NT) xAx[e] = p.xAxis[e];
        for (int e = tid; e < BR; e += NT) yAx[e] = p.yAxis[Ry * e + band];
    }
    if (I8) {
        const short* gy = p.hgY + (size_t)pol * G * H;
        for (int e = tid; e < G * BR; e += NT) {
            const int n = e / BR, r = e - n * BR;
            hyB[e] = (float)gy[(size_t)n * H + Ry * r + band];
        }
        if (tid == 0) {
            tc::mbarInitTc(bars);
            tc::mbarInitTc(bars + 1);
        }
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(tc::sAddr(tmemSlot)) : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        tc::fenceBeforeSync();
    }
    // the int16 scale: merge of every band's statistics, in band order
    if (QUANT && tid == 0) {
        const StatF* part = a.part + (size_t)unit * Ry;
        StatF tot = part[0];
        for (int b = 1; b < Ry; b++) statMerge(tot, part[b].maxI, part[b].maxIdx, part[b].P, part[b].cx, part[b].cy,
                                              part[b].cyw, part[b].e4);
        const float sc = (float)(32767.0 / (double)sqrtf(tot.maxI));
        if (band == 0) {
            const int S = p.statsStride;
            float* s = p.stats;
            const int col = pol * S + frame;
            const int per = P * S;
            s[0 * per + col] = tot.P;
            s[1 * per + col] = tot.cx / tot.P;
            s[2 * per + col] = tot.cy / tot.P;
            s[3 * per + col] = sc;
            s[4 * per + col] = __int_as_float(tot.maxIdx);
            s[5 * per + col] = p.dA * (tot.P * tot.P / tot.e4);
            s[6 * per + col] = tot.cyw / tot.P;
        }
        red[0].maxI = sc;
    }
    __syncthreads();
    float scale = 0.f;
    if (QUANT) scale = red[0].maxI;
    uint32_t tmem = 0;
    if (I8) {
        tc::fenceAfterSync();
        tmem = *tmemSlot;
    }

    // column stage: window column c = slot, outputs s at Ab[s][c]
    if (slot < w) {
        const float2* win = p.window + (size_t)unit * w * h;
        float2 v[16];
#pragma unroll
        for (int m1 = 0; m1 < 16; m1++) {
            const int j = (4 * m1 + lq - r0) & 63;
            v[m1] = j < h ? cmul(__ldg(&win[(size_t)j * w + slot]), colTw[j]) : make_float2(0.f, 0.f);
        }
        ifft64q(v, lq, tw64p);
        const int s2 = 16 * brev2(lq);
#pragma unroll
        for (int s1 = 0; s1 < 16; s1++) Ab[(s1 + s2) * AW + slot] = v[s1];
    }   // w is a multiple of 8: a warp's eight slots all take part, or none
    __syncthreads();

    // row stage: pass ps covers rows 16 ps .. 16 ps + 15 of the band, slot =
    // 8 (row - 16 ps) + v; lane quad lq holds t = s1 + 16 brev2(lq), x = 8 t + v
    const float yShift = fabsf((p.yAxis[1] - p.yAxis[0]) * (float)H);
    const float inv = (float)(1.0 / ((double)W * (double)H));
    const size_t fieldOff = (size_t)unit * W * H;
    const float K14 = (float)(1.0 / (16383.0 * 16383.0));
    const float* refF = p.refWaveF + (size_t)pol * 2 * (W + H);
    StatF st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int v = slot & (RX - 1);
    const int t2 = 16 * brev2(lq);
    bool ok = true;
    for (int ps = 0; ps < NPASS; ps++) {
        const int rl = slot >> 3;               // row within the pass
        const int rowb = ROWS_PP * ps + rl;     // row within the band (s)
        const int y = Ry * rowb + band;
        float2 vv[16];
#pragma unroll
        for (int m1 = 0; m1 < 16; m1++) {
            const int c = (4 * m1 + lq - sx0) & 63;
            vv[m1] = c < w ? cmul(Ab[rowb * AW + c], rowTw[v * AW + c]) : make_float2(0.f, 0.f);
        }
        if (I8 && ps == NPASS - 1) {
            // Ab is read for the last time: Hx takes its place
            __syncthreads();
            if (tid == 0) {
                tc::fenceProxyAsync();
                const unsigned bytes = (unsigned)(GN * WF);
                const unsigned char* src = a.hx + (size_t)pol * 2 * bytes;
                tc::mbarExpectTxTc(bars, 2 * bytes);
                tc::bulkLoad(hxHi, src, bytes, bars);
                tc::bulkLoad(hxLo, src + bytes, bytes, bars);
            }
        }
        ifft64q(vv, lq, tw64p);
        if (!QUANT) {
            // statistics over the untilted field (digHolo.cpp:8866-8870)
            const float yv = yAx[rowb];
            const float yw = yv + (yv < 0.f ? yShift : 0.f);
            float Prow = 0.f, cxrow = 0.f, e4 = 0.f;
#pragma unroll
            for (int s1 = 0; s1 < 16; s1++) {
                const int x = RX * (s1 + t2) + v;
                const float I0 = fmaf(vv[s1].x, vv[s1].x, vv[s1].y * vv[s1].y);
                const float I = I0 * inv;
                const int idx = 2 * y * W + x;
                if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
                Prow += I;
                cxrow = fmaf(xAx[x], I, cxrow);
                e4 = fmaf(I, I, e4);
            }
            st.P += Prow;
            st.cx += cxrow;
            st.cy = fmaf(yv, Prow, st.cy);
            st.cyw = fmaf(yw, Prow, st.cyw);
            st.e4 += e4;
            continue;
        }
        // reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833)
        const int2 ry = refY[rowb];
        uint32_t* srow = stage + rl * WF;
#pragma unroll
        for (int s1 = 0; s1 < 16; s1++) {
            const int x = RX * (s1 + t2) + v;
            const uint32_t rx = refX[x];
            const int xr = (int)(short)(rx & 0xFFFFu), xi = (int)(short)(rx >> 16);
            const float adjR = (float)(ry.x * xr - ry.y * xi) * K14;
            const float adjI = (float)(ry.x * xi + ry.y * xr) * K14;
            const float2 av = vv[s1];
            const float vr = __fsub_rn(__fmul_rn(av.y, adjI), __fmul_rn(av.x, adjR));
            const float vi = __fadd_rn(__fmul_rn(av.x, adjI), __fmul_rn(av.y, adjR));
            const short sr = roundSat16(scale * vr), si = roundSat16(scale * vi);
            srow[stagePhys(x)] = (uint32_t)(unsigned short)sr | ((uint32_t)(unsigned short)si << 16);
            if (p.field32) {
                const float2 rxf = make_float2(__ldg(&refF[x]), __ldg(&refF[W + x]));
                const float2 ryf = make_float2(__ldg(&refF[2 * W + y]), __ldg(&refF[2 * W + H + y]));
                const float2 wv = cmul(av, cmul(ryf, rxf));
                p.field32[fieldOff + (size_t)y * W + x] = make_float2(-wv.x, wv.y);
            }
        }
        __syncthreads();
        // the pass's 16 rows out: 8 columns per task, 16-byte stores of the
        // int16 planes, and the bytes of the overlap operand
        for (int task = tid; task < ROWS_PP * (WF / 8); task += NT) {
            const int r = task / (WF / 8), x0 = 8 * (task - r * (WF / 8));
            const uint4* src = reinterpret_cast<const uint4*>(stage + r * WF + stagePhys(x0));
            const uint4 q0 = src[0], q1 = src[1];
            const uint4 R = make_uint4(__byte_perm(q0.x, q0.y, 0x5410), __byte_perm(q0.z, q0.w, 0x5410),
                                       __byte_perm(q1.x, q1.y, 0x5410), __byte_perm(q1.z, q1.w, 0x5410));
            const uint4 Iq = make_uint4(__byte_perm(q0.x, q0.y, 0x7632), __byte_perm(q0.z, q0.w, 0x7632),
                                        __byte_perm(q1.x, q1.y, 0x7632), __byte_perm(q1.z, q1.w, 0x7632));
            const int yy = Ry * (ROWS_PP * ps + r) + band;
            const size_t o = fieldOff + (size_t)yy * W + x0;
            *reinterpret_cast<uint4*>(p.fieldR + o) = R;
            *reinterpret_cast<uint4*>(p.fieldI + o) = Iq;
            if (I8) {
                const int rowR = ROWS_PP * ps + r, rowI = BR + rowR;
                // low bytes (unsigned) and high bytes (signed) of 8 int16 values
                const uint2 rl8 = make_uint2(__byte_perm(R.x, R.y, 0x6420), __byte_perm(R.z, R.w, 0x6420));
                const uint2 rh8 = make_uint2(__byte_perm(R.x, R.y, 0x7531), __byte_perm(R.z, R.w, 0x7531));
                const uint2 il8 = make_uint2(__byte_perm(Iq.x, Iq.y, 0x6420), __byte_perm(Iq.z, Iq.w, 0x6420));
                const uint2 ih8 = make_uint2(__byte_perm(Iq.x, Iq.y, 0x7531), __byte_perm(Iq.z, Iq.w, 0x7531));
                *reinterpret_cast<uint2*>(hiPlane + planeOff(128, rowR, x0)) = rh8;
                *reinterpret_cast<uint2*>(loPlane + planeOff(128, rowR, x0)) = rl8;
                *reinterpret_cast<uint2*>(hiPlane + planeOff(128, rowI, x0)) = ih8;
                *reinterpret_cast<uint2*>(loPlane + planeOff(128, rowI, x0)) = il8;
            }
        }
        __syncthreads();
    }

    if (!QUANT) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float mI = __shfl_xor_sync(0xffffffffu, st.maxI, off);
            const int mIdx = __shfl_xor_sync(0xffffffffu, st.maxIdx, off);
            statMerge(st, mI, mIdx, __shfl_xor_sync(0xffffffffu, st.P, off), __shfl_xor_sync(0xffffffffu, st.cx, off),
                      __shfl_xor_sync(0xffffffffu, st.cy, off), __shfl_xor_sync(0xffffffffu, st.cyw, off),
                      __shfl_xor_sync(0xffffffffu, st.e4, off));
        }
        if ((tid & 31) == 0) red[warp] = st;
        __syncthreads();
        if (tid == 0) {
            StatF tot = red[0];
            for (int i = 1; i < NT / 32; i++) {
                const StatF o = red[i];
                statMerge(tot, o.maxI, o.maxIdx, o.P, o.cx, o.cy, o.cyw, o.e4);
            }
            a.part[(size_t)unit * Ry + band] = tot;
        }
        return;
    }
    if (!I8) return;

    // overlap: T[row][m] = sum_x F[row][x] Hx[m][x], rows 0..63 R, 64..127 I
    tc::fenceProxyAsync();   // the operand bytes were written by ordinary stores
    __syncthreads();
    if (tid == 0) {
        const bool loaded = tc::mbarWaitTc(bars, 0u);
        tc::fenceAfterSync();
        if (loaded) {
            const uint32_t aH = tc::sAddr(hiPlane), aL = tc::sAddr(loPlane);
            const uint32_t bH = tc::sAddr(hxHi), bL = tc::sAddr(hxLo);
            const uint32_t dSS = instrDescI8s(128, GN, true, true), dSU = instrDescI8s(128, GN, true, false);
            const uint32_t dUS = instrDescI8s(128, GN, false, true), dUU = instrDescI8s(128, GN, false, false);
            const uint32_t tHH = tmem, tMix = tmem + GN, tLL = tmem + 2 * GN;
#pragma unroll
            for (int atom = 0; atom < WF / 128; atom++) {
#pragma unroll
                for (int ks = 0; ks < 4; ks++) {
                    const uint32_t ao = (uint32_t)atom * 128 * 128 + (uint32_t)ks * 32;
                    const uint32_t bo = (uint32_t)atom * GN * 128 + (uint32_t)ks * 32;
                    const uint32_t acc = (atom > 0 || ks > 0) ? 1u : 0u;
                    mmaI8(tHH, tc::smemDesc(aH + ao), tc::smemDesc(bH + bo), dSS, acc);
                    mmaI8(tMix, tc::smemDesc(aH + ao), tc::smemDesc(bL + bo), dSU, acc);
                    mmaI8(tMix, tc::smemDesc(aL + ao), tc::smemDesc(bH + bo), dUS, 1u);
                    mmaI8(tLL, tc::smemDesc(aL + ao), tc::smemDesc(bL + bo), dUU, acc);
                }
            }
        } else if (p.status) {
            *(volatile int*)p.status = 2;
            __threadfence_system();
        }
        // a commit with nothing pending still arrives, so no thread waits in vain
        tc::mmaCommit(bars + 1);
    }
    ok = !__syncthreads_or(!tc::mbarWaitTc(bars + 1, 0u));
    tc::fenceAfterSync();
    constexpr int TLD = GN + 1;
    if (warp < 4) {
        const int row = warp * 32 + (tid & 31);
        const uint32_t rowAddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < GN; c0 += 16) {
            uint32_t hh[16], mx[16], ll[16];
            tmemLoad16u(rowAddr + (uint32_t)c0, hh);
            tmemLoad16u(rowAddr + (uint32_t)(GN + c0), mx);
            tmemLoad16u(rowAddr + (uint32_t)(2 * GN + c0), ll);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const double T = 65536.0 * (double)(int)hh[i] + 256.0 * (double)(int)mx[i] + (double)(int)ll[i];
                Tsm[row * TLD + c0 + i] = (float)T;
            }
        }
    }
    tc::fenceBeforeSync();
    __syncthreads();
    if (warp == 0) {
        tc::fenceAfterSync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem) : "memory");
    }
    if (!ok) {
        if (tid == 0 && p.status) {
            *(volatile int*)p.status = 2;
            __threadfence_system();
        }
        return;
    }
    // c_mn partial = sum over the band's rows of Hy[n][y] T[row][m]
    float2* pc = a.partCoefs + ((size_t)unit * Ry + band) * M;
    for (int mode = tid; mode < M; mode += NT) {
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2, m = g - n;
        const float* hn = hyB + n * BR;
        float cr = 0.f, ci = 0.f;
#pragma unroll 8
        for (int r = 0; r < BR; r++) {
            cr = fmaf(hn[r], Tsm[r * TLD + m], cr);
            ci = fmaf(hn[r], Tsm[(BR + r) * TLD + m], ci);
        }
        pc[mode] = make_float2(cr, ci);
    }
}

// Hx of every polarisation as bytes in the operand layout: rows m < maxMG the
// modes' int16 values, rows up to GN zero; high (signed) bytes, then low.
__global__ void k_band64_prep_hx(DhInvParams p, int GN, unsigned char* out) {
    const int G = p.maxMG;
    const int total = p.polCount * GN * WF;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int pol = e / (GN * WF), rem = e - pol * GN * WF;
        const int m = rem / WF, x = rem - m * WF;
        const int val = m < G ? (int)p.hgX[((size_t)pol * G + m) * WF + x] : 0;
        const int atom = x >> 7, chunk = (x & 127) >> 4;
        const size_t off = (size_t)atom * GN * 128 + (size_t)m * 128 + (size_t)((chunk ^ (m & 7)) << 4) + (x & 15);
        unsigned char* b = out + (size_t)pol * 2 * GN * WF;
        b[off] = (unsigned char)((val >> 8) & 0xFF);
        b[(size_t)GN * WF + off] = (unsigned char)(val & 0xFF);
    }
}

// Sum of the bands' partial coefficients, times sx[m] sy[n] / scale.
__global__ void k_band64_coefs(DhInvParams p, const float2* __restrict__ part, int nb) {
    const int P = p.polCount, M = p.modeCount, G = p.maxMG, S = p.statsStride;
    const int total = p.frameCount * P * M;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int unit = e / M, mode = e % M;
        const int pol = unit % P, frame = unit / P;
        float cr = 0.f, ci = 0.f;
        for (int b = 0; b < nb; b++) {
            const float2 v = part[((size_t)unit * nb + b) * M + mode];
            cr += v.x;
            ci += v.y;
        }
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2, m = g - n;
        const float scale = p.stats[3 * P * S + pol * S + frame];
        const float fieldScale = 1.0f / scale;
        const float ms = (float)((double)p.hgScaleX[pol * G + m] * (double)p.hgScaleY[pol * G + n] * (double)fieldScale);
        p.coefs[(size_t)frame * P * M + (size_t)pol * M + mode] = make_float2(cr * ms, ci * ms);
    }
}

struct B64Plan {
    int Ry, GN, pass;
    size_t smemStats, smemQuant;
    size_t offPart, offCoefs, offHx, scratch;
};

// cudaErrorNotSupported outside the kernel's shapes: full-resolution fields
// 512 wide and 64 to 4096 high, IFFT windows of at most 64 x 64 (sides
// multiples of 16), no overlap or the tensor-core overlap with maxMG <= 32.
cudaError_t planB64(const DhInvParams& p, int overlapKind, B64Plan& pl) {
    // a reference-wave calibration is applied by k_field_big, not here
    if (p.lowres || p.refCal) return cudaErrorNotSupported;
    const int W = 1 << p.logW, H = 1 << p.logH;
    if (W != WF || H < 64 || H > TW_N) return cudaErrorNotSupported;
    if (p.w < 16 || p.h < 16 || p.w > 64 || p.h > 64 || p.w % 16 || p.h % 16) return cudaErrorNotSupported;
    for (int q = 0; q < p.polCount; q++)
        if (p.sx0[q] < 0) return cudaErrorNotSupported;
    const bool ov = p.maxMG > 0 && p.coefs;
    if (ov && (overlapKind != 0 || p.maxMG > GNMAX)) return cudaErrorNotSupported;
    pl.Ry = H / 64;
    pl.GN = ov ? (p.maxMG <= 16 ? 16 : 32) : 16;
    pl.pass = ov ? P_I8 : P_QUANT;
    pl.smemStats = band64Smem(P_STATS, p.w, 0, 16).total;
    pl.smemQuant = band64Smem(pl.pass, p.w, ov ? p.maxMG : 0, pl.GN).total;
    if (pl.smemStats > 227 * 1024 || pl.smemQuant > 227 * 1024) return cudaErrorNotSupported;
    const size_t units = (size_t)p.frameCount * p.polCount;
    pl.offPart = 0;
    pl.offCoefs = (units * pl.Ry * sizeof(StatF) + 255) / 256 * 256;
    pl.offHx = pl.offCoefs + (ov ? (units * pl.Ry * p.modeCount * sizeof(float2) + 255) / 256 * 256 : 0);
    pl.scratch = pl.offHx + (ov ? (size_t)p.polCount * 2 * pl.GN * WF : 0);
    return cudaSuccess;
}

template <int PASS, int GN>
cudaError_t launchB64(const DhInvParams& p, const B64Args& a, size_t smem, unsigned blocks, cudaStream_t s) {
    auto kern = k_band64<PASS, GN>;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(kern), (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<blocks, NT, smem, s>>>(p, a);
    return cudaGetLastError();
}

}  // namespace

// Scratch the kernels need for this launch (0 where they do not apply).
size_t dh_field_band64_scratch_bytes(const DhInvParams& p, int overlapKind) {
    B64Plan pl;
    if (planB64(p, overlapKind, pl) != cudaSuccess) return 0;
    return pl.scratch;
}

// Full-resolution 512-wide fields by bands: statistics pass, quantising pass
// (with the exact integer overlap on the tensor cores when maxMG > 0), then
// the coefficient sum.  *overlapUsed: 0 none, 3 integer tensor cores.
cudaError_t dh_launch_field_band64(const DhInvParams& p, int overlapKind, void* scratch, size_t scratchBytes,
                                   int* overlapUsed, cudaStream_t s) {
    *overlapUsed = 0;
    B64Plan pl;
    cudaError_t e = planB64(p, overlapKind, pl);
    if (e != cudaSuccess) return e;
    if (p.frameCount * p.polCount <= 0) return cudaSuccess;
    if (!scratch || scratchBytes < pl.scratch || (reinterpret_cast<uintptr_t>(scratch) & 255)) return cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(p.fieldR) & 15) || (reinterpret_cast<uintptr_t>(p.fieldI) & 15))
        return cudaErrorNotSupported;
    unsigned char* sc = static_cast<unsigned char*>(scratch);
    B64Args a;
    a.part = reinterpret_cast<StatF*>(sc + pl.offPart);
    a.partCoefs = reinterpret_cast<float2*>(sc + pl.offCoefs);
    a.hx = sc + pl.offHx;
    const unsigned blocks = (unsigned)(p.frameCount * p.polCount * pl.Ry);
    if (pl.pass == P_I8) {
        const int total = p.polCount * pl.GN * WF;
        k_band64_prep_hx<<<(total + 255) / 256, 256, 0, s>>>(p, pl.GN, sc + pl.offHx);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((e = launchB64<P_STATS, 16>(p, a, pl.smemStats, blocks, s)) != cudaSuccess) return e;
    if (pl.pass == P_QUANT) {
        e = launchB64<P_QUANT, 16>(p, a, pl.smemQuant, blocks, s);
    } else {
        e = pl.GN == 16 ? launchB64<P_I8, 16>(p, a, pl.smemQuant, blocks, s)
                        : launchB64<P_I8, 32>(p, a, pl.smemQuant, blocks, s);
    }
    if (e != cudaSuccess) return e;
    if (pl.pass == P_I8) {
        const int total = p.frameCount * p.polCount * p.modeCount;
        int g = (total + 255) / 256;
        if (g > 148 * 16) g = 148 * 16;
        k_band64_coefs<<<g, 256, 0, s>>>(p, a.partCoefs, pl.Ry);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        *overlapUsed = 3;
    }
    return cudaSuccess;
}
