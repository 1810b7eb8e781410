// Inverse stage for full-resolution fields (IFFTResolutionMode 0): the
// Fourier window placed in the H x W plane -> IFFT -> field statistics ->
// reference wave, -conj, int16 rounding (k_field_full), then the separable HG
// overlap on the int16 field, either fused into k_field_full on the tensor
// cores (split-BF16) or by k_overlap_f32 on the CUDA cores.  Same results as k_inverse in full-resolution mode and
// as the reference's FFTW c2c backward digHolo.cpp:8734, digHoloFieldAnalysis
// digHolo.cpp:2354, applyTilt16 digHolo.cpp:2701-2837 and
// overlapFieldSeparable16 digHolo.cpp:2149-2341.
//
// Pruned IFFT: only the h x w window is non-zero.  Along y, the window rows
// sit at row_j = (r0 + j) mod H; with y = (H/h) t + u the column transform
// of column c splits into H/h independent h-point inverse FFTs
//   A[(H/h) t + u][c] = IFFT_h( b_u )[t],  b_u[row_j mod h] = win[j][c] e^{2 pi i row_j u / H},
// and along x in the same way with W/w w-point inverse FFTs per row.  Each
// thread owns 32 pixels of the field in registers (two w = 16 tasks or one
// w = 32 task) until the block has the field maximum.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"
#include "dh_fft.cuh"
#include "dh_tc.cuh"

using namespace dh;


// W, H: FFT window (= field) size; WW: IFFT window size (h = w = WW);
// OVL: fuse the split-BF16 tensor-core overlap (H = 128, maxMG <= GN).
// blockDim.x = H * W / 32; one block per (frame, polarisation).
template <int W, int H, int WW, bool OVL, int GN>
__global__ void __launch_bounds__(H * W / 32, 1) k_field_full(DhInvParams p) {
    constexpr int LOG = ilog2F(WW);
    constexpr int TX = W / WW, TY = H / WW;
    constexpr int TPT = 32 / WW;                    // stage-2 tasks per thread
    constexpr int NT = H * W / 32;
    constexpr int ALD = WW + 1;                     // stage-1 buffer row stride (complex)
    constexpr int SLD = W + 8;                      // int16 staging row stride (elements)
    constexpr int TLD = H + 1;
    extern __shared__ float4 smf4[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(smf4);
    // overlap operands first (1024-byte aligned for the 128-byte swizzle)
    unsigned char* base =
        OVL ? reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm) + 1023) & ~static_cast<uintptr_t>(1023)) : sm;
    constexpr uint32_t PB = OVL ? H * W * 2 : 0;    // one bf16 piece of one plane
    constexpr uint32_t BB = OVL ? GN * W * 2 : 0;   // one bf16 piece of Hx
    unsigned char* aHi = base;
    unsigned char* aLo = aHi + PB;
    unsigned char* bHi = aLo + PB;
    unsigned char* bLo = bHi + BB;
    float2* A = reinterpret_cast<float2*>(bLo + BB);                  // [H][ALD]
    short* sR = reinterpret_cast<short*>(A + H * ALD);                // [H][SLD]
    short* sI = sR + H * SLD;
    constexpr int TWLD = WW + 1;                    // padded: lanes with different u hit different banks
    float2* tw1 = reinterpret_cast<float2*>(sI + H * SLD);           // [TY][TWLD] e^{2 pi i row_k u / H}
    float2* tw2 = tw1 + TY * TWLD;                                     // [TX][TWLD] e^{2 pi i col_k u / W}
    float* xax = reinterpret_cast<float*>(tw2 + TX * TWLD);          // [W]
    int* refX = reinterpret_cast<int*>(xax + W);                      // [W] packed (xr, xi)
    StatF* red = reinterpret_cast<StatF*>(refX + W);                  // [NT / 32]
    float* T = reinterpret_cast<float*>(red + NT / 32);               // OVL: [2][GN][TLD]
    float* hy = T + (OVL ? 2 * GN * TLD : 0);                         // OVL: [G][TLD]
    int* modeMN = reinterpret_cast<int*>(hy + (OVL ? p.maxMG * TLD : 0));
    uint64_t* bar = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(modeMN + (OVL ? p.modeCount : 0)) + 7) & ~static_cast<uintptr_t>(7));
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bar + 1);

    const int unit = blockIdx.x;
    const int P = p.polCount;
    const int pol = unit % P, frame = unit / P;
    const int tid = threadIdx.x, warp = tid >> 5;
    const short* ref = p.refWave + (size_t)pol * 2 * (W + H);
    const int r0 = ((p.sy[pol] + H / 2) % H + H) % H;
    const int sx0 = p.sx0[pol];
    for (int x = tid; x < W; x += NT) {
        xax[x] = p.xAxis[x];
        refX[x] = ((int)(unsigned short)ref[x]) | ((int)ref[W + x] << 16);
    }
    // twiddles of the decimated sub-transforms: input k of sub-problem u
    for (int e = tid; e < TY * WW; e += NT) {
        const int u = e / WW, k = e % WW;
        const int row = (r0 + ((k - r0) & (WW - 1))) & (H - 1);
        tw1[u * TWLD + k] = expPos(p.twiddle, row * u, H);
    }
    for (int e = tid; e < TX * WW; e += NT) {
        const int u = e / WW, k = e % WW;
        const int col = (sx0 + ((k - sx0) & (WW - 1))) & (W - 1);
        tw2[u * TWLD + k] = expPos(p.twiddle, col * u, W);
    }
    const int G = p.maxMG, M = p.modeCount;
    if (OVL) {
        // Hx of this polarisation as the B operand (rows m >= G zero), Hy, modes
        for (int e = tid; e < GN * (W / 8); e += NT) {
            const int m = e / (W / 8), q = e % (W / 8);
            uint4 raw = make_uint4(0, 0, 0, 0);
            if (m < G) raw = __ldg(reinterpret_cast<const uint4*>(p.hgX + ((size_t)pol * G + m) * W) + q);
            uint4 hi, lo;
            tc::split8(raw, hi, lo);
            const uint32_t off = tc::swzOffset(GN, m, q);
            *reinterpret_cast<uint4*>(bHi + off) = hi;
            *reinterpret_cast<uint4*>(bLo + off) = lo;
        }
        for (int e = tid; e < G * H; e += NT) hy[(e / H) * TLD + (e % H)] = (float)p.hgY[(size_t)pol * G * H + e];
        for (int mode = tid; mode < M; mode += NT) {
            int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
            while ((g + 1) * (g + 2) / 2 <= mode) g++;
            while (g * (g + 1) / 2 > mode) g--;
            const int n = mode - g * (g + 1) / 2;
            modeMN[mode] = ((g - n) << 16) | n;
        }
        if (tid == 0) tc::mbarInitTc(bar);
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(tc::sAddr(tmemSlot)) : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        tc::fenceProxyAsync();
        tc::fenceBeforeSync();
    }
    __syncthreads();

    // stage 1: columns c < WW, u < TY
    const float2* win = p.window + (size_t)unit * WW * WW;
    for (int task = tid; task < WW * TY; task += NT) {
        const int c = task % WW, u = task / WW;
        float2 b[WW];
#pragma unroll
        for (int k = 0; k < WW; k++) {
            const int j = (k - r0) & (WW - 1);
            b[k] = cmul(__ldg(&win[j * WW + c]), tw1[u * TWLD + k]);
        }
        ifftDIFf<WW>(b);
#pragma unroll
        for (int i = 0; i < WW; i++) A[(TY * brevF<LOG>(i) + u) * ALD + c] = b[i];
    }
    __syncthreads();

    // stage 2: rows y < H, u < TX; the field stays in registers
    float2 f[TPT][WW];
    int ty[TPT], tu[TPT];
#pragma unroll
    for (int q = 0; q < TPT; q++) {
        const int task = tid + NT * q;
        const int y = task / TX, u = task % TX;
        ty[q] = y;
        tu[q] = u;
#pragma unroll
        for (int k = 0; k < WW; k++) {
            const int c = (k - sx0) & (WW - 1);
            f[q][k] = cmul(A[y * ALD + c], tw2[u * TWLD + k]);
        }
        ifftDIFf<WW>(f[q]);
    }

    // statistics over the untilted field (digHolo.cpp:8866-8870)
    const float yShift = fabsf((p.yAxis[1] - p.yAxis[0]) * (float)H);
    const float inv = (float)(1.0 / ((double)W * (double)H));
    StatF st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < TPT; q++) {
        const int y = ty[q];
        const float yv = p.yAxis[y];
        const float yw = yv + (yv < 0.f ? yShift : 0.f);
        float Prow = 0.f, cxrow = 0.f, e4 = 0.f;
#pragma unroll
        for (int i = 0; i < WW; i++) {
            const int x = TX * brevF<LOG>(i) + tu[q];
            const float2 a = f[q][i];
            const float I0 = fmaf(a.x, a.x, a.y * a.y);
            const float I = I0 * inv;
            const int idx = 2 * y * W + x;
            if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
            Prow += I;
            cxrow = fmaf(xax[x], I, cxrow);
            e4 = fmaf(I, I, e4);
        }
        st.P += Prow;
        st.cx += cxrow;
        st.cy = fmaf(yv, Prow, st.cy);
        st.cyw = fmaf(yw, Prow, st.cyw);
        st.e4 += e4;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float mI = __shfl_xor_sync(0xffffffffu, st.maxI, off);
        const int mIdx = __shfl_xor_sync(0xffffffffu, st.maxIdx, off);
        statMerge(st, mI, mIdx, __shfl_xor_sync(0xffffffffu, st.P, off), __shfl_xor_sync(0xffffffffu, st.cx, off),
                  __shfl_xor_sync(0xffffffffu, st.cy, off), __shfl_xor_sync(0xffffffffu, st.cyw, off),
                  __shfl_xor_sync(0xffffffffu, st.e4, off));
    }
    if ((tid & 31) == 0) red[tid >> 5] = st;
    __syncthreads();
    StatF tot = red[0];
    for (int i = 1; i < NT / 32; i++) {
        const StatF o = red[i];
        statMerge(tot, o.maxI, o.maxIdx, o.P, o.cx, o.cy, o.cyw, o.e4);
    }
    const float scale = (float)(32767.0 / (double)sqrtf(tot.maxI));
    if (tid == 0) {
        const int S = p.statsStride;
        float* s = p.stats;
        const int col = pol * S + frame;
        const int per = P * S;
        s[0 * per + col] = tot.P;
        s[1 * per + col] = tot.cx / tot.P;
        s[2 * per + col] = tot.cy / tot.P;
        s[3 * per + col] = scale;
        s[4 * per + col] = __int_as_float(tot.maxIdx);
        s[5 * per + col] = p.dA * (tot.P * tot.P / tot.e4);
        s[6 * per + col] = tot.cyw / tot.P;
    }

    // reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833)
    const float K = (float)(1.0 / (16383.0 * 16383.0));
    const size_t fieldOff = (size_t)unit * W * H;
#pragma unroll
    for (int q = 0; q < TPT; q++) {
        const int y = ty[q];
        const int yr = ref[2 * W + y], yi = ref[2 * W + H + y];
#pragma unroll
        for (int i = 0; i < WW; i++) {
            const int x = TX * brevF<LOG>(i) + tu[q];
            const int rx = refX[x];
            const int xr = (short)(rx & 0xFFFF), xi = rx >> 16;
            const float adjR = (float)(yr * xr - yi * xi) * K;
            const float adjI = (float)(yr * xi + yi * xr) * K;
            const float2 a = f[q][i];
            const float vr = __fsub_rn(__fmul_rn(a.y, adjI), __fmul_rn(a.x, adjR));
            const float vi = __fadd_rn(__fmul_rn(a.x, adjI), __fmul_rn(a.y, adjR));
            if (p.field32) {
                const float* rf = p.refWaveF + (size_t)pol * 2 * (W + H);
                const float2 rxf = make_float2(rf[x], rf[W + x]);
                const float2 ryf = make_float2(rf[2 * W + y], rf[2 * W + H + y]);
                const float2 w = cmul(a, cmul(ryf, rxf));
                p.field32[fieldOff + (size_t)y * W + x] = make_float2(-w.x, w.y);
            }
            sR[y * SLD + x] = roundSat16(scale * vr);
            sI[y * SLD + x] = roundSat16(scale * vi);
        }
    }
    if (!OVL && p.fieldsOnly) return;   // block-uniform
    __syncthreads();
    // coalesced copy of the int16 planes
    constexpr int CH = W / 8;   // 16-byte chunks per row
    uint4* gR = reinterpret_cast<uint4*>(p.fieldR + fieldOff);
    uint4* gI = reinterpret_cast<uint4*>(p.fieldI + fieldOff);
    for (int e = tid; e < H * CH; e += NT) {
        const int y = e / CH, q = e % CH;
        gR[e] = *reinterpret_cast<const uint4*>(sR + y * SLD + 8 * q);
        gI[e] = *reinterpret_cast<const uint4*>(sI + y * SLD + 8 * q);
    }
    if (!OVL) return;

    // Fused overlap (digHolo.cpp:2149-2341) on the tensor cores, split-BF16:
    // T[y][m] = sum_x V[y][x] Hx[m][x] per plane (hi.hi + hi.lo + lo.hi, FP32
    // accumulation in tensor memory), then c_mn = sum_y Hy[n][y] T[y][m].
    const uint32_t tmem = *tmemSlot;
    constexpr uint32_t IDESC = tc::instrDesc(128, GN);
    bool ok = true;
    for (int plane = 0; plane < 2 && ok; plane++) {
        const short* sp = plane ? sI : sR;
        for (int e = tid; e < H * CH; e += NT) {
            const int y = e / CH, q = e % CH;
            uint4 hi, lo;
            tc::split8(*reinterpret_cast<const uint4*>(sp + y * SLD + 8 * q), hi, lo);
            const uint32_t off = tc::swzOffset(H, y, q);
            *reinterpret_cast<uint4*>(aHi + off) = hi;
            *reinterpret_cast<uint4*>(aLo + off) = lo;
        }
        tc::fenceProxyAsync();
        __syncthreads();
        if (tid == 0) {
            tc::fenceAfterSync();
            const uint32_t d = tmem + (uint32_t)(plane * GN);
            const uint32_t aH = tc::sAddr(aHi), aL = tc::sAddr(aLo), bH = tc::sAddr(bHi), bL = tc::sAddr(bLo);
#pragma unroll
            for (int k = 0; k < W / 16; k++) {
                const uint32_t ka = (uint32_t)(k >> 2) * H * 128 + (uint32_t)(k & 3) * 32;
                const uint32_t kb = (uint32_t)(k >> 2) * GN * 128 + (uint32_t)(k & 3) * 32;
                tc::mmaBf16(d, tc::smemDesc(aH + ka), tc::smemDesc(bH + kb), IDESC, k > 0 ? 1u : 0u);
                tc::mmaBf16(d, tc::smemDesc(aH + ka), tc::smemDesc(bL + kb), IDESC, 1u);
                tc::mmaBf16(d, tc::smemDesc(aL + ka), tc::smemDesc(bH + kb), IDESC, 1u);
            }
            tc::mmaCommit(bar);
        }
        // the operand buffer is rewritten for the next plane only after the MMAs finish
        ok = !__syncthreads_or(!tc::mbarWaitTc(bar, (unsigned)plane));
        tc::fenceAfterSync();
    }
    if (ok) {
        if (warp < 4) {
            const uint32_t rowAddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
            for (int pl = 0; pl < 2; pl++) {
#pragma unroll
                for (int c0 = 0; c0 < GN; c0 += 16) {
                    float v[16];
                    tc::tmemLoad16(rowAddr + (uint32_t)(pl * GN + c0), v);
#pragma unroll
                    for (int i = 0; i < 16; i++) T[(pl * GN + c0 + i) * TLD + tid] = v[i];
                }
            }
        }
        tc::fenceBeforeSync();
        __syncthreads();
        const float fieldScale = 1.0f / scale;
        const float* sxp = p.hgScaleX + pol * G;
        const float* syp = p.hgScaleY + pol * G;
        for (int mode = tid; mode < M; mode += NT) {
            const int mn = modeMN[mode];
            const int m = mn >> 16, n = mn & 0xFFFF;
            const float* hn = hy + n * TLD;
            const float* tr = T + m * TLD;
            const float* ti = T + (GN + m) * TLD;
            float cr = 0.f, ci = 0.f;
#pragma unroll 8
            for (int yy = 0; yy < H; yy++) {
                cr = fmaf(hn[yy], tr[yy], cr);
                ci = fmaf(hn[yy], ti[yy], ci);
            }
            const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
            p.coefs[(size_t)frame * P * M + (size_t)pol * M + mode] = make_float2(cr * ms, ci * ms);
        }
    } else if (tid == 0 && p.status) {
        *(volatile int*)p.status = 2;
        __threadfence_system();
    }
    tc::fenceBeforeSync();
    __syncthreads();
    if (warp == 0) {
        tc::fenceAfterSync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
    }
}

// Separable overlap of int16 fields on the CUDA cores (FP32 accumulation):
// T[y][m] = sum_x F[y][x] Hx[m][x] with one thread per (row, plane) and the
// modes in registers, then c_mn = sum_y Hy[n][y] T[y][m] per mode.
// One block per (frame, polarisation); blockDim.x = 2 * ny.
template <int GMAX>
__global__ void __launch_bounds__(256) k_overlap_f32(DhInvParams p, int nx, int ny) {
    extern __shared__ float smo[];
    const int G = p.maxMG, M = p.modeCount;
    const int unit = blockIdx.x;
    const int P = p.polCount;
    const int pol = unit % P, frame = unit / P;
    const int tid = threadIdx.x;
    float* hx = smo;                                   // [nx][GMAX] (x-major: one float4 row per x)
    float* hy = hx + nx * GMAX;                        // [G][ny]
    float* T = hy + G * ny;                            // [2][ny][G + 1]
    const short* gx = p.hgX + (size_t)pol * G * nx;
    const short* gy = p.hgY + (size_t)pol * G * ny;
    for (int e = tid; e < nx * GMAX; e += blockDim.x) {
        const int x = e / GMAX, m = e % GMAX;
        hx[e] = m < G ? (float)gx[m * nx + x] : 0.f;
    }
    for (int e = tid; e < G * ny; e += blockDim.x) hy[e] = (float)gy[e];
    __syncthreads();
    const size_t npix = (size_t)nx * ny;
    {
        const int plane = tid / ny, y = tid % ny;
        const short* row = (plane ? p.fieldI : p.fieldR) + (size_t)unit * npix + (size_t)y * nx;
        float acc[GMAX];
#pragma unroll
        for (int m = 0; m < GMAX; m++) acc[m] = 0.f;
        for (int x0 = 0; x0 < nx; x0 += 8) {
            const uint4 raw = __ldg(reinterpret_cast<const uint4*>(row + x0));
            const unsigned wv[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const float v = (float)(short)((wv[t >> 1] >> (16 * (t & 1))) & 0xFFFF);
                const float4* hv = reinterpret_cast<const float4*>(hx + (x0 + t) * GMAX);
#pragma unroll
                for (int m4 = 0; m4 < GMAX / 4; m4++) {
                    const float4 h = hv[m4];
                    acc[4 * m4 + 0] = fmaf(v, h.x, acc[4 * m4 + 0]);
                    acc[4 * m4 + 1] = fmaf(v, h.y, acc[4 * m4 + 1]);
                    acc[4 * m4 + 2] = fmaf(v, h.z, acc[4 * m4 + 2]);
                    acc[4 * m4 + 3] = fmaf(v, h.w, acc[4 * m4 + 3]);
                }
            }
        }
        float* Tp = T + ((size_t)plane * ny + y) * (G + 1);
#pragma unroll
        for (int m = 0; m < GMAX; m++)
            if (m < G) Tp[m] = acc[m];   // unrolled: acc stays in registers
    }
    __syncthreads();
    const int S = p.statsStride;
    const float scale = p.stats[3 * P * S + pol * S + frame];
    const float fieldScale = 1.0f / scale;
    const float* sxp = p.hgScaleX + pol * G;
    const float* syp = p.hgScaleY + pol * G;
    for (int mode = tid; mode < M; mode += blockDim.x) {
        int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((g + 1) * (g + 2) / 2 <= mode) g++;
        while (g * (g + 1) / 2 > mode) g--;
        const int n = mode - g * (g + 1) / 2;
        const int m = g - n;
        const float* hn = hy + n * ny;
        float cr = 0.f, ci = 0.f;
        for (int y = 0; y < ny; y++) {
            cr = fmaf(hn[y], T[(size_t)y * (G + 1) + m], cr);
            ci = fmaf(hn[y], T[((size_t)ny + y) * (G + 1) + m], ci);
        }
        const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
        p.coefs[(size_t)frame * P * M + (size_t)pol * M + mode] = make_float2(cr * ms, ci * ms);
    }
}

// The same overlap for any number of mode groups: the x-modes in chunks of
// OVC (T[y][m] of one chunk in shared memory, the int16 field re-read per
// chunk), then c_mn for the modes whose m falls in the chunk, with Hy read
// from global memory.  Per chunk the sums run in k_overlap_f32's order, so
// the coefficients equal its bit for bit.  The fallback beyond the
// register-tiled overlaps (more than 64 mode groups, or more than 32 on
// fields taller than 128 rows).  One block of 256 threads per (frame,
// polarisation).
constexpr int OVC = 16;
__global__ void __launch_bounds__(256) k_overlap_f32_chunked(DhInvParams p, int nx, int ny) {
    extern __shared__ float smo[];
    const int G = p.maxMG, M = p.modeCount;
    const int unit = blockIdx.x;
    const int P = p.polCount;
    const int pol = unit % P, frame = unit / P;
    const int tid = threadIdx.x;
    float* hx = smo;                                   // [nx][OVC]
    float* T = hx + (size_t)nx * OVC;                  // [2][ny][OVC + 1]
    const short* gx = p.hgX + (size_t)pol * G * nx;
    const short* gy = p.hgY + (size_t)pol * G * ny;
    const size_t npix = (size_t)nx * ny;
    const int S = p.statsStride;
    const float fieldScale = 1.0f / p.stats[3 * P * S + pol * S + frame];
    const float* sxp = p.hgScaleX + pol * G;
    const float* syp = p.hgScaleY + pol * G;
    for (int m0 = 0; m0 < G; m0 += OVC) {
        __syncthreads();   // the previous chunk's tables are consumed
        for (int e = tid; e < nx * OVC; e += blockDim.x) {
            const int x = e / OVC, m = m0 + e % OVC;
            hx[e] = m < G ? (float)gx[(size_t)m * nx + x] : 0.f;
        }
        __syncthreads();
        for (int r = tid; r < 2 * ny; r += blockDim.x) {
            const int plane = r / ny, y = r - plane * ny;
            const short* row = (plane ? p.fieldI : p.fieldR) + (size_t)unit * npix + (size_t)y * nx;
            float acc[OVC];
#pragma unroll
            for (int m = 0; m < OVC; m++) acc[m] = 0.f;
            for (int x0 = 0; x0 < nx; x0 += 8) {
                const uint4 raw = __ldg(reinterpret_cast<const uint4*>(row + x0));
                const unsigned wv[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const float v = (float)(short)((wv[t >> 1] >> (16 * (t & 1))) & 0xFFFF);
                    const float4* hv = reinterpret_cast<const float4*>(hx + (x0 + t) * OVC);
#pragma unroll
                    for (int m4 = 0; m4 < OVC / 4; m4++) {
                        const float4 h = hv[m4];
                        acc[4 * m4 + 0] = fmaf(v, h.x, acc[4 * m4 + 0]);
                        acc[4 * m4 + 1] = fmaf(v, h.y, acc[4 * m4 + 1]);
                        acc[4 * m4 + 2] = fmaf(v, h.z, acc[4 * m4 + 2]);
                        acc[4 * m4 + 3] = fmaf(v, h.w, acc[4 * m4 + 3]);
                    }
                }
            }
            float* Tp = T + (size_t)r * (OVC + 1);
#pragma unroll
            for (int m = 0; m < OVC; m++) Tp[m] = acc[m];
        }
        __syncthreads();
        for (int mode = tid; mode < M; mode += blockDim.x) {
            int g = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
            while ((g + 1) * (g + 2) / 2 <= mode) g++;
            while (g * (g + 1) / 2 > mode) g--;
            const int n = mode - g * (g + 1) / 2;
            const int m = g - n;
            if (m < m0 || m >= m0 + OVC) continue;
            const short* hn = gy + (size_t)n * ny;
            const float* t0 = T + (m - m0);
            const float* t1 = T + (size_t)ny * (OVC + 1) + (m - m0);
            float cr = 0.f, ci = 0.f;
            for (int y = 0; y < ny; y++) {
                const float hv = (float)hn[y];
                cr = fmaf(hv, t0[(size_t)y * (OVC + 1)], cr);
                ci = fmaf(hv, t1[(size_t)y * (OVC + 1)], ci);
            }
            const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
            p.coefs[(size_t)frame * P * M + (size_t)pol * M + mode] = make_float2(cr * ms, ci * ms);
        }
    }
}

namespace {

template <int W, int H, int WW, bool OVL, int GN>
cudaError_t launchField(const DhInvParams& p, cudaStream_t s) {
    constexpr int NT = H * W / 32;
    const size_t ovl = OVL ? 1024 + 2 * (size_t)H * W * 2 + 2 * (size_t)GN * W * 2 : 0;
    const size_t tail = OVL ? sizeof(float) * (2 * (size_t)GN * (H + 1) + (size_t)p.maxMG * (H + 1)) +
                                  sizeof(int) * (size_t)p.modeCount + 32
                            : 0;
    const size_t smem = ovl + sizeof(float2) * (size_t)H * (WW + 1) + sizeof(short) * 2 * (size_t)H * (W + 8) +
                        sizeof(float2) * (size_t)(H / WW + W / WW) * (WW + 1) + sizeof(float) * W + sizeof(int) * W +
                        sizeof(StatF) * (NT / 32) + tail;
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    auto kern = k_field_full<W, H, WW, OVL, GN>;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(kern), (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)(p.frameCount * p.polCount), NT, smem, s>>>(p);
    return cudaGetLastError();
}

template <int GMAX>
cudaError_t launchOverlapF32(const DhInvParams& p, int nx, int ny, cudaStream_t s) {
    const size_t smem = sizeof(float) * ((size_t)nx * GMAX + (size_t)p.maxMG * ny + 2 * (size_t)ny * (p.maxMG + 1));
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_overlap_f32<GMAX>), (int)smem);
    if (e != cudaSuccess) return e;
    k_overlap_f32<GMAX><<<(unsigned)(p.frameCount * p.polCount), 2 * ny, smem, s>>>(p, nx, ny);
    return cudaGetLastError();
}

}  // namespace

// Full-resolution field kernel; cudaErrorNotSupported outside its shapes.
// withOverlap: fuse the split-BF16 tensor-core overlap (128-row fields,
// maxMG <= 32); *fused reports whether it did.
cudaError_t dh_launch_field_full(const DhInvParams& p, int withOverlap, int* fused, cudaStream_t s) {
    *fused = 0;
    if (p.lowres || p.logw != p.logh || p.logW != p.logH) return cudaErrorNotSupported;
    if (p.w != (1 << p.logw) || p.h != (1 << p.logh)) return cudaErrorNotSupported;   // power-of-two windows only
    if (p.frameCount * p.polCount <= 0) return cudaSuccess;
    const int W = 1 << p.logW, w = 1 << p.logw;
    const bool ovl = withOverlap && p.maxMG > 0 && p.coefs && p.maxMG <= 32 && W == 128;
    if (ovl) {
        *fused = 1;
        const bool small = p.maxMG <= 16;
        if (w == 16) return small ? launchField<128, 128, 16, true, 16>(p, s) : launchField<128, 128, 16, true, 32>(p, s);
        if (w == 32) return small ? launchField<128, 128, 32, true, 16>(p, s) : launchField<128, 128, 32, true, 32>(p, s);
        *fused = 0;
        return cudaErrorNotSupported;
    }
    if (w == 16) {
        if (W == 128) return launchField<128, 128, 16, false, 16>(p, s);
        if (W == 64) return launchField<64, 64, 16, false, 16>(p, s);
        if (W == 32) return launchField<32, 32, 16, false, 16>(p, s);
    } else if (w == 32) {
        if (W == 128) return launchField<128, 128, 32, false, 16>(p, s);
        if (W == 64) return launchField<64, 64, 32, false, 16>(p, s);
    }
    return cudaErrorNotSupported;
}

// FP32 overlap of the int16 fields [unit][ny][nx]; cudaErrorNotSupported
// outside its shapes (2 ny <= 256 threads, nx a multiple of 8, G <= 64).
cudaError_t dh_launch_overlap_f32(const DhInvParams& p, int nx, int ny, cudaStream_t s) {
    if (p.maxMG <= 0 || !p.coefs) return cudaSuccess;
    if (2 * ny > 256 || nx % 8 != 0 || ny < 16) return cudaErrorNotSupported;
    if (p.maxMG <= 16) return launchOverlapF32<16>(p, nx, ny, s);
    if (p.maxMG <= 32) return launchOverlapF32<32>(p, nx, ny, s);
    if (p.maxMG <= 64) return launchOverlapF32<64>(p, nx, ny, s);
    return cudaErrorNotSupported;
}

// The chunked FP32 overlap (any maxMG); cudaErrorNotSupported when nx is not
// a multiple of 8 or the chunk tables exceed shared memory.
cudaError_t dh_launch_overlap_f32_chunked(const DhInvParams& p, int nx, int ny, cudaStream_t s) {
    if (p.maxMG <= 0 || !p.coefs) return cudaSuccess;
    if (nx % 8 != 0 || nx < 8 || ny < 1) return cudaErrorNotSupported;
    const size_t smem = sizeof(float) * ((size_t)nx * OVC + 2 * (size_t)ny * (OVC + 1));
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(k_overlap_f32_chunked), (int)smem);
    if (e != cudaSuccess) return e;
    k_overlap_f32_chunked<<<(unsigned)(p.frameCount * p.polCount), 256, smem, s>>>(p, nx, ny);
    return cudaGetLastError();
}
