// Inverse stage for full-resolution fields of any size (IFFTResolutionMode 0)
// whose field does not fit one thread block: the Fourier window placed in
// the H x W plane -> IFFT -> field statistics -> reference wave, -conj,
// int16 rounding, then the separable HG overlap.  Same results as the
// reference's FFTW c2c backward digHolo.cpp:8734, digHoloFieldAnalysis
// digHolo.cpp:2354, applyTilt16 digHolo.cpp:2701-2837 and
// overlapFieldSeparable16 digHolo.cpp:2149-2341.
//
// Pruned, folded IFFT with 16-point sub-transforms.  Along y, window row j
// sits at k-space row r0 + j; with y = (H/16) s + u,
//   A[(H/16) s + u][c] = IFFT_16(b_u)[s],
//   b_u[k] = e^{2 pi i (r0 + j0) u / H} sum_f win[j0 + 16 f][c] e^{2 pi i 16 f u / H},
// j0 = (k - r0) mod 16, so every window height that is a multiple of 16 folds
// onto the same 16-point transform; along x in the same way per row.
//
// A block owns 64 rows of one field (four column sub-problems u); one field
// takes H / 64 blocks ("bands").  The field maximum that sets the int16 scale
// spans all bands, so the field is computed twice: the statistics pass
// writes one partial record per band, the quantising pass merges them (in
// band order, identically in every block), recomputes the band, writes the
// int16 planes and contracts them with Hx: on the tensor cores in
// split-BF16 (hi.hi + hi.lo + lo.hi, FP32 accumulation in tensor memory) or
// on the CUDA cores in FP32.  The K order of that contraction is the order in
// which the sub-transforms produce x (x = (W/16) brev4(i) + u), and Hx is
// prepared in the same order.  A last kernel sums the per-band partial
// coefficients c_mn = sum_y Hy[n][y] T[y][m] and applies the mode scales.
#include <cuda_bf16.h>
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

constexpr int SL = 16;    // sub-transform length
constexpr int BR = 64;    // field rows per block (2 x 64 = 128 operand rows)
constexpr int NT = 512;   // threads per block
constexpr int GNMAX = 32; // Hx rows in the contraction (maxMG <= 32)

enum { PASS_STATS = 0, PASS_QUANT = 1, PASS_TC = 2, PASS_F32 = 3 };

struct BigArgs {
    StatF* part;                 // [unit][band] partial statistics
    float2* partCoefs;           // [unit][band][modeCount]
    const unsigned char* hxTc;   // [pol][hi, lo][W / 64 atoms][GN][128 B] (swizzled bf16)
    const float* hxF;            // [pol][W][GN]
    int KR;                      // contraction K per round (64, 128 or 256)
};

__device__ __forceinline__ int brev4(int i) {
    return ((i & 1) << 3) | ((i & 2) << 1) | ((i & 4) >> 1) | ((i & 8) >> 3);
}

__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

// Exact bf16 hi + lo of 8 integers held as floats.
__device__ __forceinline__ void split8f(const float (&v)[8], uint4& hi, uint4& lo) {
    unsigned h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        const __nv_bfloat162 lb = __floats2bfloat162_rn(v[2 * i] - __low2float(hb), v[2 * i + 1] - __high2float(hb));
        h[i] = *reinterpret_cast<const unsigned*>(&hb);
        l[i] = *reinterpret_cast<const unsigned*>(&lb);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ void modeToMN(int mode, int& m, int& n) {
    int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
    while ((g + 1) * (g + 2) / 2 <= mode) g++;
    while (g * (g + 1) / 2 > mode) g--;
    n = mode - g * (g + 1) / 2;
    m = g - n;
}

// Shared-memory plan of one block; the host computes the same numbers.
struct BigSmem {
    size_t op, ab, tabs, hy, red, total;
};
__host__ __device__ inline BigSmem bigSmem(int pass, int KR, int w, int h, int G) {
    const int UR = KR / SL, Fx = w / SL, Fy = h / SL;
    const int RS = KR + KR / SL + 1;
    BigSmem s;
    s.op = pass == PASS_TC ? 1024 + (size_t)KR * 512 + (size_t)KR * GNMAX * 4
         : pass == PASS_F32 ? (size_t)128 * RS * 4 + (size_t)KR * GNMAX * 4
                            : 0;
    s.ab = sizeof(float2) * (size_t)BR * (w + 1);
    s.tabs = sizeof(float2) * (size_t)(4 * SL + 4 * Fy + UR * (SL + 1) + UR * Fx);
    s.hy = (pass == PASS_TC || pass == PASS_F32) ? sizeof(float) * (size_t)G * BR : 0;
    s.red = sizeof(StatF) * (NT / 32);
    s.total = s.op + s.ab + s.tabs + s.hy + s.red + 8 + 16 + 8;
    return s;
}

// One block: 64 rows (band) of one (frame, polarisation) field.
template <int PASS, int GN>
__global__ void __launch_bounds__(NT, 1) k_field_big(DhInvParams p, BigArgs a) {
    constexpr bool QUANT = PASS != PASS_STATS;
    constexpr bool TC = PASS == PASS_TC;
    constexpr bool F32 = PASS == PASS_F32;
    constexpr bool OV = TC || F32;
    const int W = 1 << p.logW, H = 1 << p.logH, w = p.w, h = p.h;
    const int TXc = W / SL, TYc = H / SL;
    const int nb = H / BR;
    const int Fx = w / SL, Fy = h / SL;
    const int KR = a.KR, UR = KR / SL;
    const int RS = KR + KR / SL + 1;
    const int ALD = w + 1;
    const int unit = blockIdx.x / nb, band = blockIdx.x % nb;
    const int P = p.polCount, pol = unit % P, frame = unit / P;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int G = OV ? p.maxMG : 0, M = p.modeCount;

    const BigSmem L = bigSmem(PASS, KR, w, h, G);
    extern __shared__ float4 smf4[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(smf4);
    unsigned char* base =
        TC ? reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm) + 1023) & ~static_cast<uintptr_t>(1023)) : sm;
    unsigned char* aHi = base;                              // TC: [KR / 64][128][128 B]
    unsigned char* aLo = aHi + (size_t)KR * 256;
    unsigned char* bHi = aLo + (size_t)KR * 256;            // TC: [KR / 64][GN][128 B]
    unsigned char* bLo = bHi + (size_t)KR * GN * 2;
    float* fOp = reinterpret_cast<float*>(base);            // F32: [128][RS]
    float* hxs = fOp + 128 * RS;                            // F32: [KR][GN]
    float* Tsm = reinterpret_cast<float*>(base);            // OV, after the last round: [128][GN + 1]
    float2* Ab = reinterpret_cast<float2*>(sm + L.op);      // [64][w + 1] column-stage output
    float2* cBase = Ab + BR * ALD;                          // [4][16]
    float2* cRot = cBase + 4 * SL;                          // [4][Fy]
    float2* xBase = cRot + 4 * Fy;                          // [UR][17]
    float2* xRot = xBase + UR * (SL + 1);                   // [UR][Fx]
    float* hyB = reinterpret_cast<float*>(xRot + UR * Fx);  // OV: [G][64]
    StatF* red = reinterpret_cast<StatF*>(hyB + G * BR);    // [NT / 32]
    uint64_t* bar = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(red + NT / 32) + 7) & ~static_cast<uintptr_t>(7));   // TC: load, MMA
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bar + 2);

    const int r0 = ((p.sy[pol] + H / 2) % H + H) % H;
    const int sx0 = p.sx0[pol];
    const int yBase = 4 * band;   // column sub-problems yBase .. yBase + 3

    // block row r <-> field row y = TYc (r & 15) + yBase + (r >> 4)
    for (int e = tid; e < 4 * SL; e += NT) {
        const int sub = e / SL, k = e % SL;
        const int j0 = (k - r0) & (SL - 1);
        cBase[e] = expPos(p.twiddle, (r0 + j0) * (yBase + sub), H);
    }
    for (int e = tid; e < 4 * Fy; e += NT) {
        const int sub = e / Fy, f = e % Fy;
        cRot[e] = expPos(p.twiddle, SL * f * (yBase + sub), H);
    }
    if (OV) {
        const short* gy = p.hgY + (size_t)pol * G * H;
        for (int e = tid; e < G * BR; e += NT) {
            const int n = e / BR, r = e % BR;
            hyB[e] = (float)gy[(size_t)n * H + TYc * (r & 15) + yBase + (r >> 4)];
        }
    }
    if (TC) {
        if (tid == 0) {
            tc::mbarInitTc(bar);
            tc::mbarInitTc(bar + 1);
        }
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(tc::sAddr(tmemSlot)) : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        tc::fenceBeforeSync();
    }
    // the int16 scale: merge of all bands' statistics, in band order
    float scale = 0.f;
    if (QUANT && tid == 0) {
        const StatF* part = a.part + (size_t)unit * nb;
        StatF tot = part[0];
        for (int b = 1; b < nb; b++) statMerge(tot, part[b].maxI, part[b].maxIdx, part[b].P, part[b].cx, part[b].cy,
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
    if (QUANT) scale = red[0].maxI;
    uint32_t tmem = 0;
    if (TC) {
        tc::fenceAfterSync();
        tmem = *tmemSlot;
    }

    // column stage: 4 sub-problems x w window columns
    const float2* win = p.window + (size_t)unit * w * h;
    for (int task = tid; task < 4 * w; task += NT) {
        const int sub = task / w, c = task % w;
        float2 v[SL];
#pragma unroll
        for (int k = 0; k < SL; k++) v[k] = make_float2(0.f, 0.f);
        for (int f = 0; f < Fy; f++) {
            const float2 rot = cRot[sub * Fy + f];
#pragma unroll
            for (int k = 0; k < SL; k++) {
                const int j = ((k - r0) & (SL - 1)) + SL * f;
                v[k] = cfma(__ldg(&win[(size_t)j * w + c]), rot, v[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < SL; k++) v[k] = cmul(v[k], cBase[sub * SL + k]);
        ifftDIFf<SL>(v);
#pragma unroll
        for (int i = 0; i < SL; i++) Ab[(sub * SL + brevF<4>(i)) * ALD + c] = v[i];
    }

    // row stage, in rounds of UR consecutive row sub-problems (K = 16 UR)
    const int rowsPerPass = NT / UR;
    const int ul = tid % UR, rr = tid / UR;
    const int rounds = TXc / UR;
    const float yShift = fabsf((p.yAxis[1] - p.yAxis[0]) * (float)H);
    const float inv = (float)(1.0 / ((double)W * (double)H));
    const short* ref = p.refWave + (size_t)pol * 2 * (W + H);
    const float* refF = p.refWaveF + (size_t)pol * 2 * (W + H);
    const size_t fieldOff = (size_t)unit * W * H;
    const float K14 = (float)(1.0 / (16383.0 * 16383.0));
    StatF st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
    constexpr int MPER = GN / 4;
    float acc[F32 ? MPER : 1];
#pragma unroll
    for (int j = 0; j < (F32 ? MPER : 1); j++) acc[j] = 0.f;
    bool ok = true;

    for (int rho = 0; rho < rounds; rho++) {
        if (TC && rho > 0) {
            // the operands are rewritten only after the previous round's MMAs have read them
            ok = !__syncthreads_or(!tc::mbarWaitTc(bar + 1, (unsigned)((rho - 1) & 1))) && ok;
            tc::fenceAfterSync();
        } else {
            __syncthreads();
        }
        const int u0 = rho * UR;
        for (int e = tid; e < UR * SL; e += NT) {
            const int l = e / SL, k = e % SL;
            const int c0 = (k - sx0) & (SL - 1);
            xBase[l * (SL + 1) + k] = expPos(p.twiddle, (sx0 + c0) * (u0 + l), W);
        }
        for (int e = tid; e < UR * Fx; e += NT) {
            const int l = e / Fx, f = e % Fx;
            xRot[e] = expPos(p.twiddle, SL * f * (u0 + l), W);
        }
        if (TC && tid == 0) {
            const unsigned bytes = (unsigned)(KR * GN * 2);
            const unsigned char* src = a.hxTc + (size_t)pol * 2 * W * GN * 2 + (size_t)rho * bytes;
            tc::mbarExpectTxTc(bar, 2 * bytes);
            tc::bulkLoad(bHi, src, bytes, bar);
            tc::bulkLoad(bLo, src + (size_t)W * GN * 2, bytes, bar);
        }
        if (F32) {
            const uint4* src = reinterpret_cast<const uint4*>(a.hxF + ((size_t)pol * W + (size_t)rho * KR) * GN);
            uint4* dst = reinterpret_cast<uint4*>(hxs);
            for (int e = tid; e < KR * GN / 4; e += NT) dst[e] = __ldg(src + e);
        }
        __syncthreads();

        const int ux = u0 + ul;
        for (int r = rr; r < BR; r += rowsPerPass) {
            float2 v[SL];
#pragma unroll
            for (int k = 0; k < SL; k++) v[k] = make_float2(0.f, 0.f);
            const float2* arow = Ab + r * ALD;
            for (int f = 0; f < Fx; f++) {
                const float2 rot = xRot[ul * Fx + f];
#pragma unroll
                for (int k = 0; k < SL; k++) v[k] = cfma(arow[((k - sx0) & (SL - 1)) + SL * f], rot, v[k]);
            }
#pragma unroll
            for (int k = 0; k < SL; k++) v[k] = cmul(v[k], xBase[ul * (SL + 1) + k]);
            ifftDIFf<SL>(v);
            const int y = TYc * (r & 15) + yBase + (r >> 4);
            if (p.refCal) {
                // reference-wave calibration of the IFFT output (digHolo.cpp:8736-8758, 8770-8782)
                const float2* cal = p.refCal + ((size_t)pol * H + y) * W;
#pragma unroll
                for (int i = 0; i < SL; i++) {
                    const float2 c = __ldg(&cal[TXc * brevF<4>(i) + ux]);
                    v[i] = make_float2(__fmaf_rn(v[i].x, c.x, -__fmul_rn(v[i].y, c.y)),
                                       __fmaf_rn(v[i].x, c.y, __fmul_rn(v[i].y, c.x)));
                }
            }
            if (!QUANT) {
                // statistics over the untilted field (digHolo.cpp:8866-8870)
                const float yv = p.yAxis[y];
                const float yw = yv + (yv < 0.f ? yShift : 0.f);
                float Prow = 0.f, cxrow = 0.f, e4 = 0.f;
#pragma unroll
                for (int i = 0; i < SL; i++) {
                    const int x = TXc * brevF<4>(i) + ux;
                    const float I0 = fmaf(v[i].x, v[i].x, v[i].y * v[i].y);
                    const float I = I0 * inv;
                    const int idx = 2 * y * W + x;
                    if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
                    Prow += I;
                    cxrow = fmaf(__ldg(&p.xAxis[x]), I, cxrow);
                    e4 = fmaf(I, I, e4);
                }
                st.P += Prow;
                st.cx += cxrow;
                st.cy = fmaf(yv, Prow, st.cy);
                st.cyw = fmaf(yw, Prow, st.cyw);
                st.e4 += e4;
            } else {
                // reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833)
                const int yr = ref[2 * W + y], yi = ref[2 * W + H + y];
                float qr[SL], qi[SL];
#pragma unroll
                for (int i = 0; i < SL; i++) {
                    const int x = TXc * brevF<4>(i) + ux;
                    const int xr = __ldg(&ref[x]), xi = __ldg(&ref[W + x]);
                    const float adjR = (float)(yr * xr - yi * xi) * K14;
                    const float adjI = (float)(yr * xi + yi * xr) * K14;
                    const float2 av = v[i];
                    const float vr = __fsub_rn(__fmul_rn(av.y, adjI), __fmul_rn(av.x, adjR));
                    const float vi = __fadd_rn(__fmul_rn(av.x, adjI), __fmul_rn(av.y, adjR));
                    const short sr = roundSat16(scale * vr), si = roundSat16(scale * vi);
                    const size_t o = fieldOff + (size_t)y * W + x;
                    p.fieldR[o] = sr;
                    p.fieldI[o] = si;
                    if (p.field32) {
                        const float2 rxf = make_float2(__ldg(&refF[x]), __ldg(&refF[W + x]));
                        const float2 ryf = make_float2(refF[2 * W + y], refF[2 * W + H + y]);
                        const float2 wv = cmul(av, cmul(ryf, rxf));
                        p.field32[o] = make_float2(-wv.x, wv.y);
                    }
                    qr[i] = (float)sr;
                    qi[i] = (float)si;
                }
                if (TC) {
#pragma unroll
                    for (int half = 0; half < 2; half++) {
                        float hv[8];
                        uint4 hi, lo;
#pragma unroll
                        for (int e = 0; e < 8; e++) hv[e] = qr[8 * half + e];
                        split8f(hv, hi, lo);
                        uint32_t off = tc::swzOffset(128, r, 2 * ul + half);
                        *reinterpret_cast<uint4*>(aHi + off) = hi;
                        *reinterpret_cast<uint4*>(aLo + off) = lo;
#pragma unroll
                        for (int e = 0; e < 8; e++) hv[e] = qi[8 * half + e];
                        split8f(hv, hi, lo);
                        off = tc::swzOffset(128, BR + r, 2 * ul + half);
                        *reinterpret_cast<uint4*>(aHi + off) = hi;
                        *reinterpret_cast<uint4*>(aLo + off) = lo;
                    }
                }
                if (F32) {
#pragma unroll
                    for (int i = 0; i < SL; i++) {
                        fOp[r * RS + ul * (SL + 1) + i] = qr[i];
                        fOp[(BR + r) * RS + ul * (SL + 1) + i] = qi[i];
                    }
                }
            }
        }

        if (TC) {
            tc::fenceProxyAsync();
            __syncthreads();
            if (tid == 0) {
                const bool loaded = tc::mbarWaitTc(bar, (unsigned)(rho & 1));
                tc::fenceAfterSync();
                if (loaded) {
                    constexpr uint32_t IDESC = tc::instrDesc(128, GN);
                    const uint32_t aH = tc::sAddr(aHi), aL = tc::sAddr(aLo), bH = tc::sAddr(bHi), bL = tc::sAddr(bLo);
                    for (int k = 0; k < KR / 16; k++) {
                        const uint32_t ka = (uint32_t)(k >> 2) * 128 * 128 + (uint32_t)(k & 3) * 32;
                        const uint32_t kb = (uint32_t)(k >> 2) * GN * 128 + (uint32_t)(k & 3) * 32;
                        tc::mmaBf16(tmem, tc::smemDesc(aH + ka), tc::smemDesc(bH + kb), IDESC, (rho > 0 || k > 0) ? 1u : 0u);
                        tc::mmaBf16(tmem, tc::smemDesc(aH + ka), tc::smemDesc(bL + kb), IDESC, 1u);
                        tc::mmaBf16(tmem, tc::smemDesc(aL + ka), tc::smemDesc(bH + kb), IDESC, 1u);
                    }
                } else if (p.status) {
                    *(volatile int*)p.status = 2;
                    __threadfence_system();
                }
                // a commit with nothing pending still arrives, so no thread waits in vain
                tc::mmaCommit(bar + 1);
            }
        }
        if (F32) {
            __syncthreads();
            const int mrow = tid >> 2, mg = tid & 3;
            const float* arow = fOp + mrow * RS;
            for (int kl = 0; kl < KR; kl++) {
                const float av = arow[kl + (kl >> 4)];
                const float* hv = hxs + kl * GN + mg * MPER;
#pragma unroll
                for (int j = 0; j < MPER; j++) acc[j] = fmaf(av, hv[j], acc[j]);
            }
        }
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
            a.part[(size_t)unit * nb + band] = tot;
        }
        return;
    }
    if (!OV) return;

    constexpr int TLD = GN + 1;
    if (TC) {
        ok = !__syncthreads_or(!tc::mbarWaitTc(bar + 1, (unsigned)((rounds - 1) & 1))) && ok;
        tc::fenceAfterSync();
        if (warp < 4) {
            const uint32_t rowAddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
            for (int c0 = 0; c0 < GN; c0 += 16) {
                float vv[16];
                tc::tmemLoad16(rowAddr + (uint32_t)c0, vv);
#pragma unroll
                for (int i = 0; i < 16; i++) Tsm[(warp * 32 + (tid & 31)) * TLD + c0 + i] = vv[i];
            }
        }
        tc::fenceBeforeSync();
    } else {
        __syncthreads();   // every thread is done with the operand buffer
        const int mrow = tid >> 2, mg = tid & 3;
#pragma unroll
        for (int j = 0; j < MPER; j++) Tsm[mrow * TLD + mg * MPER + j] = acc[j];
    }
    __syncthreads();
    if (TC && warp == 0) {
        tc::fenceAfterSync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
    }
    if (!ok) {
        if (tid == 0 && p.status) {
            *(volatile int*)p.status = 2;
            __threadfence_system();
        }
        return;
    }
    float2* pc = a.partCoefs + ((size_t)unit * nb + band) * M;
    for (int mode = tid; mode < M; mode += NT) {
        int m, n;
        modeToMN(mode, m, n);
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

// Hx of every polarisation in the contraction's K order (x = (W/16) brev4(i)
// + u for K index 16 u + i), rows m >= maxMG zero: bf16 hi / lo in the
// swizzled operand layout, or FP32 [K][GN].
__global__ void k_big_prep_hx(DhInvParams p, int GN, unsigned char* outTc, float* outF) {
    const int W = 1 << p.logW, TXc = W / SL, G = p.maxMG;
    const int chunks = W / 8;
    const int total = p.polCount * chunks * GN;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int pol = e / (chunks * GN);
        const int rem = e % (chunks * GN);
        const int m = rem % GN, q = rem / GN;
        float v[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int kk = 8 * q + t;
            const int x = TXc * brev4(kk & 15) + (kk >> 4);
            v[t] = m < G ? (float)p.hgX[((size_t)pol * G + m) * W + x] : 0.f;
        }
        if (outTc) {
            uint4 hi, lo;
            split8f(v, hi, lo);
            unsigned char* b = outTc + (size_t)pol * 2 * W * GN * 2;
            const uint32_t off = tc::swzOffset(GN, m, q);
            *reinterpret_cast<uint4*>(b + off) = hi;
            *reinterpret_cast<uint4*>(b + (size_t)W * GN * 2 + off) = lo;
        }
        if (outF) {
#pragma unroll
            for (int t = 0; t < 8; t++) outF[((size_t)pol * W + 8 * q + t) * GN + m] = v[t];
        }
    }
}

// Sum of the bands' partial coefficients, times sx[m] sy[n] / scale.
__global__ void k_big_coefs(DhInvParams p, const float2* __restrict__ part, int nb) {
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
        int m, n;
        modeToMN(mode, m, n);
        const float scale = p.stats[3 * P * S + pol * S + frame];
        const float fieldScale = 1.0f / scale;
        const float ms = (float)((double)p.hgScaleX[pol * G + m] * (double)p.hgScaleY[pol * G + n] * (double)fieldScale);
        p.coefs[(size_t)frame * P * M + (size_t)pol * M + mode] = make_float2(cr * ms, ci * ms);
    }
}

struct BigPlan {
    int nb, KRstats, KR, pass, GN;
    size_t smemStats, smemQuant;
    size_t offPart, offCoefs, offHx, scratch;
};

size_t alignUp(size_t v, size_t a) { return (v + a - 1) / a * a; }

// cudaErrorNotSupported outside the kernel's shapes.
cudaError_t planBig(const DhInvParams& p, int overlapKind, BigPlan& pl) {
    if (p.lowres) return cudaErrorNotSupported;
    const int W = 1 << p.logW, H = 1 << p.logH, w = p.w, h = p.h;
    if (W < 64 || H < 64 || W > TW_N || H > TW_N || w < SL || h < SL || w > W || h > H) return cudaErrorNotSupported;
    if (w % SL || h % SL) return cudaErrorNotSupported;
    const bool ov = p.maxMG > 0 && p.coefs;
    if (ov && p.maxMG > GNMAX) return cudaErrorNotSupported;
    pl.nb = H / BR;
    pl.GN = ov ? (p.maxMG <= 16 ? 16 : 32) : 0;
    pl.KRstats = W >= 256 ? 256 : W;
    pl.smemStats = bigSmem(PASS_STATS, pl.KRstats, w, h, 0).total;
    if (pl.smemStats > 227 * 1024) return cudaErrorNotSupported;
    pl.pass = !ov ? PASS_QUANT : (overlapKind == 0 ? PASS_TC : PASS_F32);
    pl.KR = 0;
    for (int kr = 256; kr >= 64; kr >>= 1) {
        if (kr > W) continue;
        const size_t s = bigSmem(pl.pass, kr, w, h, ov ? p.maxMG : 0).total;
        if (s <= 227 * 1024) { pl.KR = kr; pl.smemQuant = s; break; }
    }
    if (pl.KR == 0) return cudaErrorNotSupported;
    const size_t units = (size_t)p.frameCount * p.polCount;
    pl.offPart = 0;
    pl.offCoefs = alignUp(units * pl.nb * sizeof(StatF), 256);
    pl.offHx = alignUp(pl.offCoefs + (ov ? units * pl.nb * p.modeCount * sizeof(float2) : 0), 256);
    pl.scratch = pl.offHx + (ov ? (size_t)p.polCount * W * GNMAX * sizeof(float) : 0);
    return cudaSuccess;
}

template <int PASS, int GN>
cudaError_t launchBand(const DhInvParams& p, const BigArgs& a, size_t smem, unsigned blocks, cudaStream_t s) {
    auto kern = k_field_big<PASS, GN>;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(kern), (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<blocks, NT, smem, s>>>(p, a);
    return cudaGetLastError();
}

}  // namespace

// Scratch the band kernels need for this launch (0 where they do not apply).
size_t dh_field_big_scratch_bytes(const DhInvParams& p, int overlapKind) {
    BigPlan pl;
    if (planBig(p, overlapKind, pl) != cudaSuccess) return 0;
    return pl.scratch;
}

// Full-resolution fields by bands: statistics pass, quantising pass (with the
// overlap: overlapKind 0 split-BF16 tensor cores, 1 FP32 CUDA cores), then the
// coefficient sum.  *overlapUsed: 0 none, 1 FP32, 2 tensor cores.
cudaError_t dh_launch_field_big(const DhInvParams& p, int overlapKind, void* scratch, size_t scratchBytes,
                                int* overlapUsed, cudaStream_t s) {
    *overlapUsed = 0;
    BigPlan pl;
    cudaError_t e = planBig(p, overlapKind, pl);
    if (e != cudaSuccess) return e;
    if (p.frameCount * p.polCount <= 0) return cudaSuccess;
    if (!scratch || scratchBytes < pl.scratch || (reinterpret_cast<uintptr_t>(scratch) & 255)) return cudaErrorInvalidValue;
    unsigned char* sc = static_cast<unsigned char*>(scratch);
    BigArgs a;
    a.part = reinterpret_cast<StatF*>(sc + pl.offPart);
    a.partCoefs = reinterpret_cast<float2*>(sc + pl.offCoefs);
    a.hxTc = sc + pl.offHx;
    a.hxF = reinterpret_cast<const float*>(sc + pl.offHx);
    const unsigned blocks = (unsigned)(p.frameCount * p.polCount * pl.nb);
    if (pl.pass == PASS_TC || pl.pass == PASS_F32) {
        const int W = 1 << p.logW;
        const int total = p.polCount * (W / 8) * pl.GN;
        k_big_prep_hx<<<(total + 255) / 256, 256, 0, s>>>(p, pl.GN, pl.pass == PASS_TC ? sc + pl.offHx : nullptr,
                                                          pl.pass == PASS_F32 ? reinterpret_cast<float*>(sc + pl.offHx) : nullptr);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    a.KR = pl.KRstats;
    if ((e = launchBand<PASS_STATS, 16>(p, a, pl.smemStats, blocks, s)) != cudaSuccess) return e;
    a.KR = pl.KR;
    if (pl.pass == PASS_QUANT) {
        e = launchBand<PASS_QUANT, 16>(p, a, pl.smemQuant, blocks, s);
    } else if (pl.pass == PASS_TC) {
        e = pl.GN == 16 ? launchBand<PASS_TC, 16>(p, a, pl.smemQuant, blocks, s)
                        : launchBand<PASS_TC, 32>(p, a, pl.smemQuant, blocks, s);
    } else {
        e = pl.GN == 16 ? launchBand<PASS_F32, 16>(p, a, pl.smemQuant, blocks, s)
                        : launchBand<PASS_F32, 32>(p, a, pl.smemQuant, blocks, s);
    }
    if (e != cudaSuccess) return e;
    if (pl.pass == PASS_TC || pl.pass == PASS_F32) {
        const int total = p.frameCount * p.polCount * p.modeCount;
        int g = (total + 255) / 256;
        if (g > 148 * 16) g = 148 * 16;
        k_big_coefs<<<g, 256, 0, s>>>(p, a.partCoefs, pl.nb);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        *overlapUsed = pl.pass == PASS_TC ? 2 : 1;
    }
    return cudaSuccess;
}
