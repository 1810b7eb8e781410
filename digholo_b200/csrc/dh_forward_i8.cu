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
// tcgen05.mma.kind::i8 products accumulate in tensor memory (int32):
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
// loads (NA stages), warp 1 the MMAs (two tensor-memory accumulator sets
// when they fit), warps 2-9 read the accumulators and run the column stage.
// Each block serves one polarisation.  Every wait is bounded; on expiry the
// kernel records the failure in p.status and leaves after its copies land.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

#include "dh_common.cuh"
#include "dh_params.h"
#include "dh_tc.cuh"
#include "dh_twiddle128.h"

using namespace dh;

namespace {

constexpr int NTHREADS = 320;   // 10 warps
constexpr int NEPI = 256;       // epilogue threads (warps 2-9)
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
__device__ __forceinline__ void epiSync() { asm volatile("bar.sync 1, %0;" ::"n"(NEPI) : "memory"); }

__device__ __forceinline__ void flagFail(const DhFwdParams& p, volatile int* abortFlag) {
    *abortFlag = 1;
    if (p.status) {
        *(volatile int*)p.status = 1;
        __threadfence_system();
    }
}

}  // namespace

// W: FFT-window width (K = 2W bytes per row), HW: IFFT window (h = w),
// NPAD: accumulator columns (2 w + ones column, rounded up to 16), NB:
// accumulator sets in tensor memory, NA: TMA stages.  H = 128 rows.
template <int W, int HW, int NPAD, int NB, int NA>
__global__ void __launch_bounds__(NTHREADS, 1) k_forward_i8(const __grid_constant__ CUtensorMap tmap, DhFwdParams p) {
    constexpr int H = MROWS;
    constexpr int KB = 2 * W;                     // bytes per row
    constexpr int NATOM = KB / 128;               // 128-byte K atoms
    constexpr unsigned ABYTES = (unsigned)H * KB; // one stage
    constexpr int BQ = NATOM * NPAD * 128;        // one accumulator's operand bytes
    constexpr int w = HW, h = HW;
    constexpr int Q = H / HW;
    constexpr int CLD = w + 1;
    constexpr int LOGHW = ilog2I(HW);
    constexpr uint32_t IDESC = instrDescI8(128, NPAD);
    constexpr int TMEMCOLS = (4 * NPAD * NB) <= 256 ? 256 : 512;

    extern __shared__ unsigned char smRaw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smRaw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* aBuf = base;                                   // [NA][NATOM][128 rows][128 B]
    unsigned char* bBuf = aBuf + (size_t)NA * ABYTES;             // [4][NATOM][NPAD][128 B]
    float2* colbuf = reinterpret_cast<float2*>(bBuf + 4 * BQ);    // [H][w + 1]
    float2* exch = colbuf + (size_t)H * CLD;                      // [HW][Q][w]
    float2* tCol = exch + (size_t)H * w;                          // [h][Q] (this polarisation)
    float2* tAdj = tCol + (size_t)h * Q;                          // [h][w]
    uint64_t* bars = reinterpret_cast<uint64_t*>(tAdj + (size_t)h * w);
    uint64_t* full = bars;                // [NA]
    uint64_t* empty = bars + NA;          // [NA]
    uint64_t* accFull = bars + 2 * NA;    // [NB]
    uint64_t* accEmpty = accFull + NB;    // [NB]
    uint64_t* bLoad = accEmpty + NB;      // the operand table
    uint64_t* drain = bLoad + 1;          // final MMA commit
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abortFlag = reinterpret_cast<volatile int*>(tmemSlot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int P = p.polCount;
    const int pol = blockIdx.x % P;
    const int frameStep = gridDim.x / P;
    const int frame0 = blockIdx.x / P;
    const int nIt = frame0 < p.frameCount ? (p.frameCount - frame0 + frameStep - 1) / frameStep : 0;

    for (int e = tid; e < h * Q; e += NTHREADS) tCol[e] = p.tabCol[(size_t)pol * h * Q + e];
    for (int e = tid; e < h * w; e += NTHREADS) tAdj[e] = p.tabAdj[(size_t)pol * h * w + e];
    if (tid == 0) {
        for (int s = 0; s < NA; s++) { mbarInitN(&full[s], 1); mbarInitN(&empty[s], 1); }
        for (int b = 0; b < NB; b++) { mbarInitN(&accFull[b], 1); mbarInitN(&accEmpty[b], 1); }
        mbarInitN(bLoad, 1);
        mbarInitN(drain, 1);
        *abortFlag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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
    const int rowsPerFrame = (int)(p.frameStride / p.frameWidth);

    if (warp == 0) {
        // ---------------- TMA producer
        if (lane == 0) {
            const unsigned char* tab = p.dftDigits + (size_t)pol * 4 * BQ;
            tc::fenceProxyAsync();
            tc::mbarExpectTxTc(bLoad, 4 * BQ);
            for (int q = 0; q < 4; q++) tc::bulkLoad(bBuf + q * BQ, tab + q * BQ, BQ, bLoad);
            int issued = 0;
            for (int it = 0; it < nIt; it++) {
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
        // ---------------- MMA issuer
        if (lane == 0) {
            bool ok = tc::mbarWaitTc(bLoad, 0);
            if (!ok) flagFail(p, abortFlag);
            for (int it = 0; ok && it < nIt; it++) {
                const int s = it % NA, b = it % NB;
                if (!tc::mbarWaitTc(&full[s], (unsigned)((it / NA) & 1))) { flagFail(p, abortFlag); break; }
                if (it >= NB && !tc::mbarWaitTc(&accEmpty[b], (unsigned)(((it / NB) - 1) & 1))) {
                    flagFail(p, abortFlag);
                    break;
                }
                if (*abortFlag) break;
                tc::fenceAfterSync();
                const uint32_t aS = tc::sAddr(aBuf + (size_t)s * ABYTES);
                const uint32_t bS = tc::sAddr(bBuf);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint32_t d = tmem + (uint32_t)(b * 4 * NPAD + q * NPAD);
#pragma unroll
                    for (int a = 0; a < NATOM; a++) {
#pragma unroll
                        for (int ks = 0; ks < 4; ks++) {
                            const uint32_t ao = (uint32_t)a * H * 128 + (uint32_t)ks * 32;
                            const uint32_t bo = (uint32_t)(q * BQ + a * NPAD * 128 + ks * 32);
                            mmaI8(d, tc::smemDesc(aS + ao), tc::smemDesc(bS + bo), IDESC, (a > 0 || ks > 0) ? 1u : 0u);
                        }
                    }
                }
                tc::mmaCommit(&empty[s]);
                tc::mmaCommit(&accFull[b]);
            }
            // every MMA issued here completes before the accumulators are freed
            tc::mmaCommit(drain);
            tc::mbarWaitTc(drain, 0);
        }
    } else {
        // ---------------- accumulator readback, column stage, output
        const int et = tid - 64;                 // 0 .. 255
        const int quarter = warp & 3;            // tensor-memory lanes 32 quarter .. + 31
        const int grp = (warp - 2) >> 2;         // 0: real columns, 1: imaginary columns
        const int r = 32 * quarter + lane;       // FFT-window row
        for (int it = 0; it < nIt; it++) {
            const int b = it % NB;
            const int frame = frame0 + it * frameStep;
            const bool okAcc = tc::mbarWaitTc(&accFull[b], (unsigned)((it / NB) & 1));
            if (!okAcc) flagFail(p, abortFlag);
            // all epilogue threads agree before touching the accumulators
            epiSync();
            if (*abortFlag) break;
            tc::fenceAfterSync();
            {
                const uint32_t rowAddr = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(b * 4 * NPAD);
                uint32_t dv[4][HW], sv[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
#pragma unroll
                    for (int c0 = 0; c0 < HW; c0 += 16) {
                        uint32_t t16[16];
                        tmemLdX<16>(rowAddr + (uint32_t)(q * NPAD + grp * w + c0), t16);
#pragma unroll
                        for (int i = 0; i < 16; i++) dv[q][c0 + i] = t16[i];
                    }
                    tmemLd1(rowAddr + (uint32_t)(q * NPAD + 2 * w), sv[q]);
                }
                tmemWaitLd();
                tc::fenceBeforeSync();
                epiSync();
                if (et == 0) mbarArrive(&accEmpty[b]);
                const long long S = ((long long)(int)sv[0] << 24) + ((long long)(int)sv[1] << 16) +
                                    ((long long)(int)sv[2] << 8) + (long long)(int)sv[3];
                const long long S22 = S << 22;
                float* cr = reinterpret_cast<float*>(colbuf + (size_t)r * CLD) + grp;
#pragma unroll
                for (int c = 0; c < HW; c++) {
                    const long long T = ((long long)(int)dv[0][c] << 24) + ((long long)(int)dv[1][c] << 16) +
                                        ((long long)(int)dv[2][c] << 8) + (long long)(int)dv[3][c];
                    cr[2 * c] = __ll2float_rn(T - S22) * 2.384185791015625e-07f;   // 2^-22
                }
            }
            epiSync();

            // column transforms of the decimated sequences X[Q a + bq][c], a < HW
            for (int e = et; e < w * Q; e += NEPI) {
                const int c = e % w, bq = e / w;
                float2 v[HW];
#pragma unroll
                for (int a = 0; a < HW; a++) v[a] = colbuf[(size_t)(Q * a + bq) * CLD + c];
                fftDIFi<HW>(v);
#pragma unroll
                for (int i = 0; i < HW; i++) exch[((size_t)brevI<LOGHW>(i) * Q + bq) * w + c] = v[i];
            }
            epiSync();

            // kept rows: Y = sum_b tCol[j][b] Z_b[row mod HW], then the window factors
            float2 bc = make_float2(1.0f, 0.0f);
            if (p.batchCal && p.batchCalCount > 0)
                bc = p.batchCal[pol * p.batchCalCount + ((p.frameOffset + frame) % p.batchCalCount)];
            const int sy = p.sy[pol];
            float2* out = p.window + (size_t)(frame * P + pol) * h * w;
            for (int e = et; e < h * w; e += NEPI) {
                const int j = e / w, c = e - j * w;
                const int row = (j + sy + H / 2) & (H - 1);
                const float2* zb = exch + (size_t)(row & (HW - 1)) * Q * w + c;
                const float2* tcj = tCol + (size_t)j * Q;
                float2 Y = zb[0];
                for (int bq = 1; bq < Q; bq++) Y = cadd(Y, cmul(zb[(size_t)bq * w], tcj[bq]));
                out[e] = cmul(cmul(Y, bc), tAdj[e]);
            }
            // the next unit rewrites colbuf only after its first barrier, and
            // exch only after its second: every thread is past this loop by then
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

PFN_cuTensorMapEncodeTiled_v12000 encodeFnI8() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

template <int W, int HW, int NPAD, int NB, int NA>
size_t smemI8() {
    const int H = MROWS, Q = H / HW;
    return 1024 + (size_t)NA * H * 2 * W + (size_t)4 * (2 * W / 128) * NPAD * 128 +
           sizeof(float2) * ((size_t)H * (HW + 1) + (size_t)H * HW + (size_t)HW * Q + (size_t)HW * HW) +
           sizeof(uint64_t) * (2 * NA + 2 * NB + 2) + 16;
}

template <int W, int HW, int NPAD, int NB, int NA>
cudaError_t launchI8(const DhFwdParams& p, const CUtensorMap& map, cudaStream_t s) {
    size_t smem = smemI8<W, HW, NPAD, NB, NA>();
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    // more than half an SM's shared memory: one block per SM, so one tensor-memory allocation per SM
    if (smem < 120 * 1024) smem = 120 * 1024;
    auto kern = k_forward_i8<W, HW, NPAD, NB, NA>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int P = p.polCount;
    // one block per SM, each serving one polarisation; at most one block per unit
    int grid = sms < p.frameCount * P ? sms : p.frameCount * P;
    grid = (grid / P) * P;
    if (grid < P) grid = P;
    kern<<<grid, NTHREADS, smem, s>>>(map, p);
    return cudaGetLastError();
}

}  // namespace

// Accumulator columns of the digit table: 2 w + 1 rounded up to 16.
int dh_forward_i8_npad(int w) { return ((2 * w + 1) + 15) / 16 * 16; }

// Returns cudaErrorNotSupported when the shape, the alignment, the digit
// table or the driver rules this kernel out (the caller then uses another
// forward kernel).
cudaError_t dh_launch_forward_i8(const DhFwdParams& p, cudaStream_t s) {
    const int W = 1 << p.logW, H = 1 << p.logH;
    if (p.frameCount <= 0) return cudaSuccess;
    if (!p.inputU16 || !p.dftDigits || !p.tabCol || !p.tabAdj) return cudaErrorNotSupported;
    if (H != MROWS || p.h != p.w || (p.w != 16 && p.w != 32)) return cudaErrorNotSupported;
    if (W != 64 && W != 128) return cudaErrorNotSupported;
    if (p.dftNpad != dh_forward_i8_npad(p.w)) return cudaErrorNotSupported;
    for (int q = 0; q < p.polCount; q++)
        if ((p.cx[q] * 2) % 16 != 0) return cudaErrorNotSupported;   // TMA x coordinate: 16-byte multiple
    if ((reinterpret_cast<uintptr_t>(p.frames) % 16) != 0 || ((size_t)p.frameWidth * 2) % 16 != 0) return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(p.dftDigits) % 16) != 0) return cudaErrorNotSupported;
    if (p.frameStride % p.frameWidth != 0) return cudaErrorNotSupported;
    const long long rowsPerFrame = p.frameStride / p.frameWidth;
    const long long totalRows = rowsPerFrame * p.frameCount;
    if (totalRows >= (1ll << 31)) return cudaErrorNotSupported;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encodeFnI8();
    if (!enc) return cudaErrorNotSupported;
    CUtensorMap map;
    const cuuint64_t dims[2] = {(cuuint64_t)p.frameWidth, (cuuint64_t)totalRows};
    const cuuint64_t strides[1] = {(cuuint64_t)p.frameWidth * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)H};
    const cuuint32_t estr[2] = {1, 1};
    CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void*>(p.frames), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorNotSupported;
    if (W == 128) {
        if (p.w == 16) return launchI8<128, 16, 48, 2, 3>(p, map, s);
        return launchI8<128, 32, 80, 1, 2>(p, map, s);
    }
    if (p.w == 16) return launchI8<64, 16, 48, 2, 4>(p, map, s);
    return launchI8<64, 32, 80, 1, 4>(p, map, s);
}
