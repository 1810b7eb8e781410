// Forward stage for uint16 frames on the tensor cores (same results as
// k_forward_tma / k_forward and the reference's FFTW r2c +
// digHoloCopyWindow, digHolo.cpp:7184-7260 and 1808-2122, to FP32 rounding).
//
// The row transform is a DFT pruned to the w kept kx columns, evaluated as an
// exact integer product on the 5th-generation tensor cores:
//
//   X[r][k] = sum_x f[r][x] e^{-2 pi i k x / W},  f = lo + 256 hi (bytes),
//
// with cos(2 pi k x / W) + 1 and -sin(2 pi k x / W) + 1 rounded to 22-bit
// fixed point v = d0 2^16 + d1 2^8 + d2 (unsigned bytes d0 <= 128).  The
// frame rows go from HBM into shared memory by TMA exactly as stored (their
// bytes are the u8 A operand, K = 2W bytes per row), and four
// tcgen05.mma.kind::i8 products accumulate in tensor memory (int32), the
// four accumulators side by side as one wide MMA per K step:
//
//   D_0 = sum hi d0,   D_1 = sum lo d0 + hi d1,   D_2 = sum lo d1 + hi d2,
//   D_3 = sum lo d2,   T = D_0 2^24 + D_1 2^16 + D_2 2^8 + D_3 = sum f v,
//
// exact in int64.  A ones column gives S = sum f, and X = (T - 2^22 S) 2^-22
// is rounded once to FP32.  The twiddles carry 22 bits, so the error is
// about the rounding of an FP32 FFT.
//
// The column transform, the window factors and the output are the TMA
// kernel's: h-point register FFTs of the H/h decimated column sequences, an
// H/h-term twiddled sum for the kept ky rows, times mask, normalisation,
// inverse pixel sinc, beam-centre phase and batch calibration.
//
// Persistent, warp-specialised, one block per SM: warp 0 issues the TMA
// loads (NA stages), warp 1 the MMAs into (up to) two tensor-memory
// accumulator sets, and NG groups of four epilogue warps take the units in turn (each
// group reads its unit's accumulators, frees them, and runs the column stage
// in its own buffer under its own named barrier), so NG units are in the
// epilogue at once.
// Each block serves one polarisation.  Every wait is bounded; on expiry the
// kernel records the failure in p.status and leaves after its copies land.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include <cstring>
#include <mutex>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"
#include "dh_tc.cuh"
#include "dh_twiddle128.h"

using namespace dh;

namespace {

constexpr int MROWS = 128;      // FFT-window rows (M of the MMA)

template <int LOG>
__host__ __device__ constexpr int brevI(int i) {
    int r = 0;
    for (int b = 0; b < LOG; b++) r |= ((i >> b) & 1) << (LOG - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2I(int n) { return n <= 1 ? 0 : 1 + ilog2I(n / 2); }

// In-place radix-2 DIF FFT of N <= 64 values in registers (natural-order
// input, bit-reversed output), exp(-2 pi i / N).
template <int N>
__device__ __forceinline__ void fftDIFi(float2 (&v)[N]) {
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
                    v[blk + j + m] = make_float2(d.y, -d.x);
                } else {
                    v[blk + j + m] = cmul(d, tw128(j * (128 / (2 * m))));
                }
            }
        }
    }
}

// In-place radix-2 DIF inverse FFT (exp(+2 pi i / N), unnormalised) of N <= 64
// values in registers: natural-order input, bit-reversed output.
template <int N>
__device__ __forceinline__ void ifftDIFi(float2 (&v)[N]) {
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
                    v[blk + j + m] = make_float2(-d.y, d.x);
                } else {
                    const float2 t = tw128(j * (128 / (2 * m)));
                    v[blk + j + m] = cmul(d, make_float2(t.x, -t.y));
                }
            }
        }
    }
}

struct StatI {
    float maxI;
    int maxIdx;
    float P, cx, cy, cyw, e4;
};

// Reduction over lanes 0 .. L-1 of one warp.
template <int L>
__device__ __forceinline__ void laneReduce(StatI& s) {
    constexpr unsigned mask = L == 32 ? 0xffffffffu : ((1u << L) - 1u);
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) {
        const float mI = __shfl_xor_sync(mask, s.maxI, off);
        const int mIdx = __shfl_xor_sync(mask, s.maxIdx, off);
        if (mI > s.maxI || (mI == s.maxI && mIdx > s.maxIdx)) { s.maxI = mI; s.maxIdx = mIdx; }
        s.P += __shfl_xor_sync(mask, s.P, off);
        s.cx += __shfl_xor_sync(mask, s.cx, off);
        s.cy += __shfl_xor_sync(mask, s.cy, off);
        s.cyw += __shfl_xor_sync(mask, s.cyw, off);
        s.e4 += __shfl_xor_sync(mask, s.e4, off);
    }
}

__device__ __forceinline__ void mbarInitN(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc::sAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::sAddr(bar)) : "memory");
}
__device__ __forceinline__ void tmaLoad2D(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            tc::sAddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(tc::sAddr(bar))
        : "memory");
}
__device__ __forceinline__ void mmaI8(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Instruction descriptor, kind::i8: u8 A and B, int32 accumulator, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t instrDescI8(int M, int N) {
    return (2u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
template <int NC>
__device__ __forceinline__ void tmemLdX(uint32_t taddr, uint32_t (&r)[NC]);
template <>
__device__ __forceinline__ void tmemLdX<16>(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmemLd1(uint32_t taddr, uint32_t& r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
}
__device__ __forceinline__ void tmemWaitLd() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Named barrier over one epilogue group (128 threads) that also returns
// whether any thread of the group passed true.
__device__ __forceinline__ bool groupSyncOr(unsigned id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void flagFail(const DhFwdParams& p, volatile int* abortFlag) {
    *abortFlag = 1;
    if (p.status) {
        *(volatile int*)p.status = 1;
        __threadfence_system();
    }
}

__host__ __device__ constexpr int dh_forward_i8_npad_impl(int w) { return ((2 * w + 1) + 7) / 8 * 8; }

__device__ __forceinline__ void groupBar(unsigned id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// Inverse stage of one unit by its epilogue group (128 threads, named
// barrier barId), for L x L low-resolution fields: the window rows and then
// columns are inverse-transformed by L threads (the last L-point transforms
// and the statistics stay inside one warp), the field is rounded to int16,
// and the separable overlap U[x][n] = sum_y Hy[n][y] V[y][x], c_mn =
// sum_x Hx[m][x] U[x][n] is spread over the group.  Radix-2 transforms as in
// k_inverse_lo<32>; the two-launch 16-pixel kernel (k_inverse_lo16q) splits
// its transforms 4 x 4 and sums in another order, so the two agree to
// rounding.  work: at least L (3 L + 3 + G) complex.
template <int L>
__device__ __forceinline__ void fusedInverse(const DhInvParams& ip, int gt, unsigned barId, int frame, int pol,
                                             const float2* winT, float2* work, float* sclSlot, const float* hxT,
                                             const float* hyT, const float* axT, const int* refT, const float* hsT) {
    constexpr int LOG = ilog2I(L);
    constexpr int LD = L + 1;
    const int P = ip.polCount, G = ip.maxMG, M = ip.modeCount;
    const int ULD = (G + 1) | 1;
    float2* t2 = work;               // [L][LD] row transforms
    float2* Vt = work + L * LD;      // [L][LD] int16 field
    float2* Ut = work + 2 * L * LD;  // [L][ULD]
    const int unit = frame * P + pol;
    groupBar(barId);   // the window tile is complete and the column buffer is free
    if (gt < L) {
        // row gt of the window, inverse FFT over kx
        float2 v[L];
#pragma unroll
        for (int c = 0; c < L; c++) v[c] = winT[gt * LD + c];
        ifftDIFi<L>(v);
#pragma unroll
        for (int i = 0; i < L; i++) t2[gt * LD + brevI<LOG>(i)] = v[i];
    }
    groupBar(barId);
    if (gt < L) {
        // column x = gt over ky: v[i] = F[y = brev(i)][x]
        const int x = gt;
        float2 v[L];
#pragma unroll
        for (int j = 0; j < L; j++) v[j] = t2[j * LD + x];
        ifftDIFi<L>(v);
        // statistics over the untilted field (digHolo.cpp:8866-8870)
        const float inv = (float)(1.0 / ((double)L * (double)L));
        const float* yax = axT + L;
        const float yShift = fabsf((yax[1] - yax[0]) * (float)L);
        const float xv = axT[x];
        StatI st = {0.f, -1, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int i = 0; i < L; i++) {
            const int y = brevI<LOG>(i);
            const float2 a = v[i];
            const float I0 = fmaf(a.x, a.x, a.y * a.y);
            const float I = I0 * inv;
            const int idx = 2 * y * L + x;
            if (I0 > st.maxI || (I0 == st.maxI && idx > st.maxIdx)) { st.maxI = I0; st.maxIdx = idx; }
            const float yv = yax[y];
            st.P += I;
            st.cx = fmaf(xv, I, st.cx);
            st.cy = fmaf(yv, I, st.cy);
            st.cyw = fmaf(yv + (yv < 0.f ? yShift : 0.f), I, st.cyw);
            st.e4 = fmaf(I, I, st.e4);
        }
        laneReduce<L>(st);
        const float scale = (float)(32767.0 / (double)sqrtf(st.maxI));
        if (x == 0) {
            const int S = ip.statsStride;
            float* sp = ip.stats;
            const int col = pol * S + frame;
            const int per = P * S;
            sp[0 * per + col] = st.P;
            sp[1 * per + col] = st.cx / st.P;
            sp[2 * per + col] = st.cy / st.P;
            sp[3 * per + col] = scale;
            sp[4 * per + col] = __int_as_float(st.maxIdx);
            sp[5 * per + col] = ip.dA * (st.P * st.P / st.e4);
            sp[6 * per + col] = st.cyw / st.P;
            *sclSlot = scale;
        }
        // reference wave, -conj(A . ref), int16 rounding (digHolo.cpp:2741-2833)
        // the wave and the scales come from shared memory: no global load
        // waits behind the field stores
        const int* ref = refT + (size_t)pol * 4 * L;
        const int xr = ref[x], xi = ref[L + x];
        const float K = (float)(1.0 / (16383.0 * 16383.0));
        const size_t fieldOff = (size_t)unit * L * L;
#pragma unroll
        for (int i = 0; i < L; i++) {
            const int y = brevI<LOG>(i);
            const int yr = ref[2 * L + y], yi = ref[3 * L + y];
            const float adjR = (float)(yr * xr - yi * xi) * K;
            const float adjI = (float)(yr * xi + yi * xr) * K;
            const float2 a = v[i];
            const float vr = __fsub_rn(__fmul_rn(a.y, adjI), __fmul_rn(a.x, adjR));
            const float vi = __fadd_rn(__fmul_rn(a.x, adjI), __fmul_rn(a.y, adjR));
            const size_t o = fieldOff + (size_t)y * L + x;
            if (ip.field32) {
                const float* rf = ip.refWaveF + (size_t)pol * 4 * L;
                const float2 rx = make_float2(rf[x], rf[L + x]);
                const float2 ry = make_float2(rf[2 * L + y], rf[3 * L + y]);
                const float2 wv = cmul(a, cmul(ry, rx));
                ip.field32[o] = make_float2(-wv.x, wv.y);
            }
            const short sr = roundSat16(scale * vr);
            const short si = roundSat16(scale * vi);
            ip.fieldR[o] = sr;
            ip.fieldI[o] = si;
            Vt[y * LD + x] = make_float2((float)sr, (float)si);
        }
    }
    if (G <= 0 || !ip.coefs) return;
    groupBar(barId);
    // overlap on the int16 field (digHolo.cpp:2149-2341), contracted over y first
    const float* hyp = hyT + (size_t)pol * G * LD;
    const float* hxp = hxT + (size_t)pol * G * LD;
    for (int e = gt; e < L * G; e += 128) {
        const int x = e % L, n = e / L;
        const float* hn = hyp + n * LD;
        float ur = 0.f, ui = 0.f;
#pragma unroll
        for (int i = 0; i < L; i++) {
            const int y = brevI<LOG>(i);
            const float hv = hn[y];
            const float2 vv = Vt[y * LD + x];
            ur = fmaf(hv, vv.x, ur);
            ui = fmaf(hv, vv.y, ui);
        }
        Ut[x * ULD + n] = make_float2(ur, ui);
    }
    groupBar(barId);
    const float fieldScale = 1.0f / *sclSlot;
    const float* sxp = hsT + pol * G;
    const float* syp = hsT + P * G + pol * G;
    float2* cout = ip.coefs + (size_t)frame * P * M + (size_t)pol * M;
    for (int mode = gt; mode < M; mode += 128) {
        int gg = (int)((sqrtf(8.0f * mode + 1.0f) - 1.0f) * 0.5f);
        while ((gg + 1) * (gg + 2) / 2 <= mode) gg++;
        while (gg * (gg + 1) / 2 > mode) gg--;
        const int n = mode - gg * (gg + 1) / 2;
        const int m = gg - n;
        const float* hm = hxp + m * LD;
        float cr = 0.f, ci = 0.f;
#pragma unroll
        for (int x = 0; x < L; x++) {
            const float2 u = Ut[x * ULD + n];
            cr = fmaf(hm[x], u.x, cr);
            ci = fmaf(hm[x], u.y, ci);
        }
        const float ms = (float)((double)sxp[m] * (double)syp[n] * (double)fieldScale);
        cout[mode] = make_float2(cr * ms, ci * ms);
    }
}

// Shared-memory plan (byte offsets from the 1024-aligned base); the host
// computes the same numbers.  FUSE adds, per epilogue group, the window
// tile and, per block, the HG tables of the fused inverse stage.
struct I8Smem {
    size_t a, b, col, tcol, tadj, win, scl, hx, hy, ax, ref, hs, bars, total;
};
__host__ __device__ inline I8Smem i8Smem(int W, int HW, int NPAD, int NA, int NG, bool fuse, int P, int G) {
    const int H = MROWS, Q = H / HW, CLD = HW + 1;
    I8Smem s;
    s.a = 0;
    s.b = s.a + (size_t)NA * H * 2 * W;
    s.col = s.b + (size_t)4 * (2 * W / 128) * NPAD * 128;
    s.tcol = s.col + sizeof(float2) * (size_t)NG * H * CLD;
    s.tadj = s.tcol + sizeof(float2) * (size_t)HW * Q;
    s.win = s.tadj + sizeof(float2) * (size_t)HW * HW;
    s.scl = s.win + (fuse ? sizeof(float2) * (size_t)NG * HW * CLD : 0);
    s.hx = s.scl + (fuse ? sizeof(float2) * (size_t)NG : 0);
    s.hy = s.hx + (fuse ? sizeof(float) * (size_t)P * G * CLD : 0);
    s.ax = s.hy + (fuse ? sizeof(float) * (size_t)P * G * CLD : 0);
    s.ref = s.ax + (fuse ? sizeof(float) * 2 * (size_t)HW : 0);
    s.hs = s.ref + (fuse ? sizeof(int) * 4 * (size_t)P * HW : 0);
    s.bars = (s.hs + (fuse ? sizeof(float) * 2 * (size_t)P * G : 0) + 7) & ~(size_t)7;
    s.total = s.bars + sizeof(uint64_t) * (2 * NA + 2 * NG + 2) + 16;
    return s;
}

}  // namespace

// W: FFT-window width (K = 2W bytes per row), HW: IFFT window (h = w),
// NPAD: accumulator columns (2 w + ones column, rounded up to 8), NA: TMA
// stages, NG: epilogue groups of four warps.  H = 128 rows; two
// tensor-memory accumulator sets where they fit (w = 16), else one.
// FUSE: the inverse stage of 16 x 16 low-resolution fields runs in the
// epilogue groups as well (window IFFT -> statistics -> reference wave,
// -conj, int16 rounding -> HG overlap; digHolo.cpp:8734, 2354, 2701-2837,
// 2149-2341), with ip its parameters.
template <int W, int HW, int NPAD, int NA, int NG, bool FUSE>
__global__ void __launch_bounds__(64 + 128 * NG, 1) k_forward_i8(const __grid_constant__ CUtensorMap tmap, DhFwdParams p,
                                                                 DhInvParams ip) {
    constexpr int H = MROWS;
    constexpr int NT = 64 + 128 * NG;
    constexpr int NB = 8 * NPAD <= 512 ? 2 : 1;   // accumulator sets
    constexpr int KB = 2 * W;                     // bytes per row
    constexpr int NATOM = KB / 128;               // 128-byte K atoms
    constexpr unsigned ABYTES = (unsigned)H * KB; // one stage
    constexpr int BQ = NATOM * NPAD * 128;        // one accumulator's operand bytes
    constexpr int w = HW, h = HW;
    constexpr int Q = H / HW;
    constexpr int CLD = w + 1;
    constexpr int LOGHW = ilog2I(HW);
    constexpr int NPART = 4 * NPAD <= 256 ? 1 : 2;  // MMAs per K step
    constexpr int NMMA = 4 * NPAD / NPART;          // their N
    static_assert(NMMA % 16 == 0 && NMMA <= 256, "MMA N must be a multiple of 16 up to 256 (M = 128)");
    constexpr uint32_t IDESC = instrDescI8(128, NMMA);
    constexpr int TMEMCOLS = 512;
    static_assert(4 * NPAD * NB <= TMEMCOLS, "accumulator sets exceed tensor memory");

    extern __shared__ unsigned char smRaw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smRaw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int GI = FUSE ? ip.maxMG : 0;
    const I8Smem L8 = i8Smem(W, HW, NPAD, NA, NG, FUSE, p.polCount, GI);
    unsigned char* aBuf = base + L8.a;                            // [NA][NATOM][128 rows][128 B]
    unsigned char* bBuf = base + L8.b;                            // [NATOM][4 NPAD][128 B]
    float2* colAll = reinterpret_cast<float2*>(base + L8.col);    // [NG][H][w + 1]
    float2* tCol = reinterpret_cast<float2*>(base + L8.tcol);     // [h][Q] (this polarisation)
    float2* tAdj = reinterpret_cast<float2*>(base + L8.tadj);     // [h][w]
    float2* winAll = reinterpret_cast<float2*>(base + L8.win);    // FUSE: [NG][h][w + 1] the unit's window
    float* sclAll = reinterpret_cast<float*>(base + L8.scl);      // FUSE: [NG] field scale
    float* hxT = reinterpret_cast<float*>(base + L8.hx);          // FUSE: [P][G][w + 1] Hx
    float* hyT = reinterpret_cast<float*>(base + L8.hy);          // FUSE: [P][G][h + 1] Hy
    float* axT = reinterpret_cast<float*>(base + L8.ax);          // FUSE: x axis [w], y axis [h]
    int* refT = reinterpret_cast<int*>(base + L8.ref);            // FUSE: [P][Xr Xi Yr Yi][16] 14-bit wave
    float* hsT = reinterpret_cast<float*>(base + L8.hs);          // FUSE: [x, y][P][G] mode scales
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + L8.bars);
    uint64_t* full = bars;                // [NA]
    uint64_t* empty = bars + NA;          // [NA]
    uint64_t* accFull = bars + 2 * NA;    // [NG] one per epilogue group
    uint64_t* accEmpty = accFull + NG;    // [NG]
    uint64_t* bLoad = accEmpty + NG;      // the operand table
    uint64_t* drain = bLoad + 1;          // final MMA commit
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abortFlag = reinterpret_cast<volatile int*>(tmemSlot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int P = p.polCount;
    const int pol = blockIdx.x % P;
    const int frameStep = gridDim.x / P;
    const int frame0 = blockIdx.x / P;
    const int nIt = frame0 < p.frameCount ? (p.frameCount - frame0 + frameStep - 1) / frameStep : 0;

    const int rowsPerFrame = (int)(p.frameStride / p.frameWidth);
    int pre = 0;   // frame tiles issued by thread 0 before the block barrier
    if (tid == 0) {
        for (int s = 0; s < NA; s++) { mbarInitN(&full[s], 1); mbarInitN(&empty[s], 1); }
        for (int g = 0; g < NG; g++) { mbarInitN(&accFull[g], 1); mbarInitN(&accEmpty[g], 1); }
        mbarInitN(bLoad, 1);
        mbarInitN(drain, 1);
        *abortFlag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // the digit table and the first NA frame tiles go out before the
        // window tables are staged and the block synchronises: their latency
        // overlaps the prologue (thread 0 is the TMA producer below)
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap)) : "memory");
        tc::fenceProxyAsync();
        tc::mbarExpectTxTc(bLoad, 4 * BQ);
        tc::bulkLoad(bBuf, p.dftDigits + (size_t)pol * 4 * BQ, 4 * BQ, bLoad);
        for (; pre < NA && pre < nIt; pre++) {
            const int frame = frame0 + pre * frameStep;
            unsigned char* dst = aBuf + (size_t)pre * ABYTES;
            tc::mbarExpectTxTc(&full[pre], ABYTES);
#pragma unroll
            for (int a = 0; a < NATOM; a++)
                tmaLoad2D(dst + (size_t)a * H * 128, &tmap, p.cx[pol] + a * 64, frame * rowsPerFrame + p.cy[pol], &full[pre]);
        }
    }
    for (int e = tid; e < h * Q; e += NT) tCol[e] = p.tabCol[(size_t)pol * h * Q + e];
    for (int e = tid; e < h * w; e += NT) tAdj[e] = p.tabAdj[(size_t)pol * h * w + e];
    if (FUSE) {
        for (int e = tid; e < P * GI * HW; e += NT) {
            const int row = e / HW, x = e - row * HW;
            hxT[row * CLD + x] = (float)ip.hgX[e];
            hyT[row * CLD + x] = (float)ip.hgY[e];
        }
        for (int e = tid; e < HW; e += NT) {
            axT[e] = ip.xAxis[e];
            axT[HW + e] = ip.yAxis[e];
        }
        for (int e = tid; e < P * 4 * HW; e += NT) refT[e] = ip.refWave[e];
        for (int e = tid; e < P * GI; e += NT) {
            hsT[e] = ip.hgScaleX[e];
            hsT[P * GI + e] = ip.hgScaleY[e];
        }
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::sAddr(tmemSlot)),
                     "n"(TMEMCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fenceBeforeSync();
    __syncthreads();
    tc::fenceAfterSync();
    const uint32_t tmem = *tmemSlot;

    if (warp == 0) {
        // ---------------- TMA producer (the first `pre` tiles are out already)
        if (lane == 0) {
            int issued = pre;
            for (int it = pre; it < nIt; it++) {
                const int s = it % NA;
                if (it >= NA && !tc::mbarWaitTc(&empty[s], (unsigned)(((it / NA) - 1) & 1))) {
                    flagFail(p, abortFlag);
                    break;
                }
                if (*abortFlag) break;
                const int frame = frame0 + it * frameStep;
                unsigned char* dst = aBuf + (size_t)s * ABYTES;
                tc::mbarExpectTxTc(&full[s], ABYTES);
#pragma unroll
                for (int a = 0; a < NATOM; a++)
                    tmaLoad2D(dst + (size_t)a * H * 128, &tmap, p.cx[pol] + a * 64, frame * rowsPerFrame + p.cy[pol], &full[s]);
                issued = it + 1;
            }
            // leave only after every copy issued here has landed
            tc::mbarWaitTc(bLoad, 0);
            for (int it = issued - NA < 0 ? 0 : issued - NA; it < issued; it++)
                tc::mbarWaitTc(&full[it % NA], (unsigned)((it / NA) & 1));
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer: unit it -> accumulator set it % 2, group it % NG
        if (lane == 0) {
            bool ok = tc::mbarWaitTc(bLoad, 0);
            if (!ok) flagFail(p, abortFlag);
            for (int it = 0; ok && it < nIt; it++) {
                const int s = it % NA, b = it % NB, g = it % NG;
                if (!tc::mbarWaitTc(&full[s], (unsigned)((it / NA) & 1))) { flagFail(p, abortFlag); break; }
                // the set was last read for unit it - 2, by group (it - 2) % NG
                if (it >= NB && !tc::mbarWaitTc(&accEmpty[(it - NB) % NG], (unsigned)(((it - NB) / NG) & 1))) {
                    flagFail(p, abortFlag);
                    break;
                }
                if (*abortFlag) break;
                tc::fenceAfterSync();
                const uint32_t aS = tc::sAddr(aBuf + (size_t)s * ABYTES);
                const uint32_t bS = tc::sAddr(bBuf);
                // the four accumulators side by side: one MMA of N = 4 NPAD per
                // K step (two of 2 NPAD where 4 NPAD exceeds 256)
#pragma unroll
                for (int part = 0; part < NPART; part++) {
                    const uint32_t d = tmem + (uint32_t)(b * 4 * NPAD + part * NMMA);
#pragma unroll
                    for (int a = 0; a < NATOM; a++) {
#pragma unroll
                        for (int ks = 0; ks < 4; ks++) {
                            const uint32_t ao = (uint32_t)a * H * 128 + (uint32_t)ks * 32;
                            const uint32_t bo = (uint32_t)(a * 4 * NPAD * 128 + part * NMMA * 128 + ks * 32);
                            mmaI8(d, tc::smemDesc(aS + ao), tc::smemDesc(bS + bo), IDESC, (a > 0 || ks > 0) ? 1u : 0u);
                        }
                    }
                }
                tc::mmaCommit(&empty[s]);
                tc::mmaCommit(&accFull[g]);
            }
            // every MMA issued here completes before the accumulators are freed
            tc::mmaCommit(drain);
            tc::mbarWaitTc(drain, 0);
        }
    } else {
        // ---------------- epilogue group g: units it = g, g + NG, ...
        const int g = (warp - 2) >> 2;
        const int gt = tid - 64 - 128 * g;       // 0 .. 127
        const int quarter = warp & 3;            // tensor-memory lanes 32 quarter .. + 31
        const int r = 32 * quarter + lane;       // FFT-window row
        const unsigned barId = 1 + g;
        float2* colbuf = colAll + (size_t)g * H * CLD;
        int k = 0;
        for (int it = g; it < nIt; it += NG, k++) {
            const int b = it % NB;
            const int frame = frame0 + it * frameStep;
            bool bad = !tc::mbarWaitTc(&accFull[g], (unsigned)(k & 1));
            if (bad) flagFail(p, abortFlag);
            // one decision for the whole group
            if (groupSyncOr(barId, bad || *abortFlag)) break;
            tc::fenceAfterSync();
            {
                // X = (D_0 4 - S) + D_1 2^-6 + D_2 2^-14 + D_3 2^-22: the first
                // difference is exact (both below 2^24), then three roundings
                const uint32_t rowAddr = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(b * 4 * NPAD);
                float xr[2 * HW];
                uint32_t s2, s3;
                tmemLd1(rowAddr + (uint32_t)(2 * NPAD + 2 * w), s2);
                tmemLd1(rowAddr + (uint32_t)(3 * NPAD + 2 * w), s3);
#pragma unroll
                for (int c0 = 0; c0 < 2 * HW; c0 += 16) {
                    uint32_t t16[16];
                    tmemLdX<16>(rowAddr + (uint32_t)c0, t16);
                    tmemWaitLd();
#pragma unroll
                    for (int i = 0; i < 16; i++) xr[c0 + i] = 4.0f * (float)(int)t16[i];
                }
                const float S = (float)((int)s2 * 256 + (int)s3);
#pragma unroll
                for (int i = 0; i < 2 * HW; i++) xr[i] -= S;
                const float scl[3] = {1.0f / 64.0f, 1.0f / 16384.0f, 1.0f / 4194304.0f};
#pragma unroll
                for (int q = 1; q < 4; q++) {
#pragma unroll
                    for (int c0 = 0; c0 < 2 * HW; c0 += 16) {
                        uint32_t t16[16];
                        tmemLdX<16>(rowAddr + (uint32_t)(q * NPAD + c0), t16);
                        tmemWaitLd();
#pragma unroll
                        for (int i = 0; i < 16; i++) xr[c0 + i] = fmaf((float)(int)t16[i], scl[q - 1], xr[c0 + i]);
                    }
                }
                tc::fenceBeforeSync();
                asm volatile("bar.sync %0, 128;" ::"r"(barId) : "memory");
                if (gt == 0) mbarArrive(&accEmpty[g]);
                float2* crow = colbuf + (size_t)r * CLD;
#pragma unroll
                for (int c = 0; c < HW; c++) crow[c] = make_float2(xr[c], xr[HW + c]);
            }
            asm volatile("bar.sync %0, 128;" ::"r"(barId) : "memory");

            // column transforms of the decimated sequences X[Q a + bq][c], a < HW,
            // in place: the outputs of (c, bq) go to the rows Q brev(i) + bq it read
            for (int e = gt; e < w * Q; e += 128) {
                const int c = e % w, bq = e / w;
                float2 v[HW];
#pragma unroll
                for (int a = 0; a < HW; a++) v[a] = colbuf[(size_t)(Q * a + bq) * CLD + c];
                fftDIFi<HW>(v);
#pragma unroll
                for (int i = 0; i < HW; i++) colbuf[(size_t)(Q * brevI<LOGHW>(i) + bq) * CLD + c] = v[i];
            }
            asm volatile("bar.sync %0, 128;" ::"r"(barId) : "memory");

            // kept rows: Y = sum_b tCol[j][b] Z_b[row mod HW], then the window factors
            float2 bc = make_float2(1.0f, 0.0f);
            if (p.batchCal && p.batchCalCount > 0)
                bc = p.batchCal[pol * p.batchCalCount + ((p.frameOffset + frame) % p.batchCalCount)];
            const int sy = p.sy[pol];
            float2* out = p.window + (size_t)(frame * P + pol) * h * w;
            for (int e = gt; e < h * w; e += 128) {
                const int j = e / w, c = e - j * w;
                const int row = (j + sy + H / 2) & (H - 1);
                const float2* zb = colbuf + (size_t)(Q * (row & (HW - 1))) * CLD + c;
                const float2* tcj = tCol + (size_t)j * Q;
                float2 Y = zb[0];
#pragma unroll
                for (int bq = 1; bq < Q; bq++) Y = cadd(Y, cmul(zb[(size_t)bq * CLD], tcj[bq]));
                const float2 wv = cmul(cmul(Y, bc), tAdj[e]);
                out[e] = wv;
                if (FUSE) winAll[(size_t)g * HW * CLD + j * CLD + c] = wv;
            }
            if (FUSE) fusedInverse<HW>(ip, gt, barId, frame, pol, winAll + (size_t)g * HW * CLD, colbuf, sclAll + g, hxT,
                                       hyT, axT, refT, hsT);
            // colbuf is rewritten for the group's next unit only after its
            // first barrier there, which every thread reaches after this loop
        }
    }

    tc::fenceBeforeSync();
    __syncthreads();
    if (warp == 1) {
        tc::fenceAfterSync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(TMEMCOLS) : "memory");
    }
}

namespace {

template <int W, int HW, int NPAD, int NA, int NG, bool FUSE>
cudaError_t launchI8(const DhFwdParams& p, const DhInvParams& ip, const CUtensorMap& map, cudaStream_t s) {
    size_t smem = 1024 + i8Smem(W, HW, NPAD, NA, NG, FUSE, p.polCount, FUSE ? ip.maxMG : 0).total;
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    // more than half an SM's shared memory: one block per SM, so one tensor-memory allocation per SM
    if (smem < 120 * 1024) smem = 120 * 1024;
    auto kern = k_forward_i8<W, HW, NPAD, NA, NG, FUSE>;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(kern), (int)smem);
    if (e != cudaSuccess) return e;
    const int sms = smCountCached();
    const int P = p.polCount;
    // one block per SM, each serving one polarisation; at most one block per unit
    int grid = sms < p.frameCount * P ? sms : p.frameCount * P;
    grid = (grid / P) * P;
    if (grid < P) grid = P;
    kern<<<grid, 64 + 128 * NG, smem, s>>>(map, p, ip);
    return cudaGetLastError();
}

// Common checks and the tensor map of the frames.
cudaError_t prepareI8(const DhFwdParams& p, CUtensorMap& map) {
    const int W = 1 << p.logW, H = 1 << p.logH;
    if (!p.inputU16 || !p.dftDigits || !p.tabCol || !p.tabAdj) return cudaErrorNotSupported;
    if (H != MROWS || p.h != p.w || (p.w != 16 && p.w != 32)) return cudaErrorNotSupported;
    if (W != 64 && W != 128) return cudaErrorNotSupported;
    if (p.dftNpad != dh_forward_i8_npad_impl(p.w)) return cudaErrorNotSupported;
    for (int q = 0; q < p.polCount; q++)
        if ((p.cx[q] * 2) % 16 != 0) return cudaErrorNotSupported;   // TMA x coordinate: 16-byte multiple
    if ((reinterpret_cast<uintptr_t>(p.frames) % 16) != 0 || ((size_t)p.frameWidth * 2) % 16 != 0) return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(p.dftDigits) % 16) != 0) return cudaErrorNotSupported;
    if (p.frameStride % p.frameWidth != 0) return cudaErrorNotSupported;
    const long long rowsPerFrame = p.frameStride / p.frameWidth;
    const long long totalRows = rowsPerFrame * p.frameCount;
    if (totalRows >= (1ll << 31)) return cudaErrorNotSupported;
    if (!frameTensorMap(map, p.frames, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, (unsigned long long)p.frameWidth,
                        (unsigned long long)totalRows, 64, (unsigned)H))
        return cudaErrorNotSupported;
    return cudaSuccess;
}

}  // namespace

// Accumulator columns of the digit table: 2 w + 1 rounded up to 8.
int dh_forward_i8_npad(int w) { return dh_forward_i8_npad_impl(w); }

// Returns cudaErrorNotSupported when the shape, the alignment, the digit
// table or the driver rules this kernel out (the caller then uses another
// forward kernel).
cudaError_t dh_launch_forward_i8(const DhFwdParams& p, cudaStream_t s) {
    if (p.frameCount <= 0) return cudaSuccess;
    CUtensorMap map;
    cudaError_t e = prepareI8(p, map);
    if (e != cudaSuccess) return e;
    DhInvParams none;
    memset(&none, 0, sizeof(none));
    const int W = 1 << p.logW;
    if (W == 128) {
        if (p.w == 16) return launchI8<128, 16, 40, 4, 3, false>(p, none, map, s);
        return launchI8<128, 32, 72, 2, 2, false>(p, none, map, s);
    }
    if (p.w == 16) return launchI8<64, 16, 40, 4, 3, false>(p, none, map, s);
    return launchI8<64, 32, 72, 4, 2, false>(p, none, map, s);
}

// Forward and inverse stages in one launch (16 x 16 low-resolution fields,
// maxMG <= 32): the frames' Fourier windows, int16 fields, statistics and
// coefficients.  cudaErrorNotSupported outside those shapes.
cudaError_t dh_launch_forward_i8_fused(const DhFwdParams& p, const DhInvParams& ip, cudaStream_t s) {
    if (!ip.lowres || ip.logw != 4 || ip.logh != 4 || p.w != 16 || ip.polCount != p.polCount) return cudaErrorNotSupported;
    if (ip.frameCount != p.frameCount || ip.maxMG > 32 || !ip.fieldR || !ip.fieldI || !ip.stats) return cudaErrorNotSupported;
    if (ip.maxMG > 0 && (!ip.hgX || !ip.hgY || !ip.hgScaleX || !ip.hgScaleY)) return cudaErrorNotSupported;
    if (p.frameCount <= 0) return cudaSuccess;
    CUtensorMap map;
    cudaError_t e = prepareI8(p, map);
    if (e != cudaSuccess) return e;
    DhInvParams q = ip;
    if (!q.coefs) q.maxMG = 0;
    if (q.maxMG <= 0) { q.maxMG = 0; q.modeCount = 0; }
    const int W = 1 << p.logW;
    if (W == 128) return launchI8<128, 16, 40, 3, 3, true>(p, q, map, s);
    return launchI8<64, 16, 40, 4, 3, true>(p, q, map, s);
}
