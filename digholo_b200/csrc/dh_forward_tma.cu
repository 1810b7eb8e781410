// Forward stage, persistent TMA-fed variant (same results as k_forward_reg
// and k_forward, and as the reference's FFTW r2c + digHoloCopyWindow,
// digHolo.cpp:7184-7260 and 1808-2122).
//
// Each block loops over (frame, polarisation) units.  The FFT window of the
// next unit is fetched by the tensor memory accelerator (2-D tiled
// cp.async.bulk.tensor, 128-byte swizzle) into the second of two shared
// buffers while the current unit is transformed, so the HBM reads overlap
// the arithmetic.  Per unit:
//
//   1. row transforms: two threads per row (warp-uniform parity), each runs
//      one half of the packed half-length complex DIF FFT in registers with
//      literal twiddles;
//   2. the R2C split is evaluated in registers for the kept kx columns only
//      (Z[k] and Z[N-k] always land in the same thread) and written to a
//      padded column buffer;
//   3. column transforms: h-point register FFTs of the H/h decimated column
//      sequences, then an H/h-term twiddled sum for the kept ky rows, times
//      the per-configuration window factors (mask, normalisation, inverse
//      pixel sinc, beam-centre phase) and the batch calibration.
//
// Every wait on a TMA completion is bounded; on expiry the kernel records
// the failure in p.status and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

#include "dh_common.cuh"
#include "dh_host.h"
#include "dh_params.h"
#include "dh_twiddle128.h"

using namespace dh;

namespace {

template <int LOG>
__host__ __device__ constexpr int brevT(int i) {
    int r = 0;
    for (int b = 0; b < LOG; b++) r |= ((i >> b) & 1) << (LOG - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2T(int n) { return n <= 1 ? 0 : 1 + ilog2T(n / 2); }

// In-place radix-2 DIF FFT of N <= 64 values in registers (natural-order
// input, bit-reversed output), exp(-2 pi i / N).
template <int N>
__device__ __forceinline__ void fftDIF(float2 (&v)[N]) {
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

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarInitFence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void proxyFence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when the phase did not complete within the limit.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < (1 << 22); i++)
        if (mbarTryWait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tmaLoad2D(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smemAddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smemAddr(bar))
        : "memory");
}

// 2^23 + u carries the integer u in its mantissa.
__device__ __forceinline__ float magicLo(unsigned int u) { return __int_as_float(0x4B000000u | (u & 0xFFFFu)); }
__device__ __forceinline__ float magicHi(unsigned int u) { return __int_as_float(0x4B000000u | (u >> 16)); }

// Packed samples 4q .. 4q+3 (uint16) or 2q .. 2q+1 (float32) of row r from
// the swizzled tile.  Tile layout: boxes of 128-byte rows, box k holds
// bytes [128k, 128k + 128) of every row; 16-byte chunk c of row r sits at
// chunk c ^ (r & 7) (the TMA 128-byte swizzle).
__device__ __forceinline__ const uint4* chunkPtr(const unsigned char* tile, int H, int r, int q) {
    const int box = q >> 3, c = q & 7;
    return reinterpret_cast<const uint4*>(tile + (size_t)box * H * 128 + r * 128 + ((c ^ (r & 7)) << 4));
}

// First DIF stage of the packed row, parity HF: HF = 0 forms s[j] + s[j+HALF]
// (the even outputs), HF = 1 forms (s[j] - s[j+HALF]) w_N^j (the odd ones).
template <int N, int HF, bool U16>
__device__ __forceinline__ void loadRow(const unsigned char* tile, int H, int r, float2 (&u)[N / 2]) {
    constexpr int HALF = N / 2;
    if (U16) {
        // 4 packed samples per chunk; s[j] with j < HALF in chunks [0, HALF/4)
#pragma unroll
        for (int q = 0; q < HALF / 4; q++) {
            const uint4 a = *chunkPtr(tile, H, r, q);
            const uint4 b = *chunkPtr(tile, H, r, q + HALF / 4);
            const unsigned aw[4] = {a.x, a.y, a.z, a.w};
            const unsigned bw[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int j = 4 * q + t;
                if (HF == 0) {
                    // (2^23 + a) + ((2^23 + b) - 2^24) = a + b exactly
                    u[j] = make_float2(magicLo(aw[t]) + (magicLo(bw[t]) - 16777216.0f),
                                       magicHi(aw[t]) + (magicHi(bw[t]) - 16777216.0f));
                } else {
                    const float2 d = make_float2(magicLo(aw[t]) - magicLo(bw[t]), magicHi(aw[t]) - magicHi(bw[t]));
                    u[j] = j == 0 ? d : cmul(d, tw128(j * (128 / N)));
                }
            }
        }
    } else {
        // 2 packed samples per chunk
#pragma unroll
        for (int q = 0; q < HALF / 2; q++) {
            const float4 a = *reinterpret_cast<const float4*>(chunkPtr(tile, H, r, q));
            const float4 b = *reinterpret_cast<const float4*>(chunkPtr(tile, H, r, q + HALF / 2));
            const float2 av[2] = {make_float2(a.x, a.y), make_float2(a.z, a.w)};
            const float2 bv[2] = {make_float2(b.x, b.y), make_float2(b.z, b.w)};
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const int j = 2 * q + t;
                if (HF == 0) u[j] = cadd(av[t], bv[t]);
                else {
                    const float2 d = csub(av[t], bv[t]);
                    u[j] = j == 0 ? d : cmul(d, tw128(j * (128 / N)));
                }
            }
        }
    }
}

// R2C split X[k] = (Z[k] + conj Z[N-k]) / 2 - i w_2N^k (Z[k] - conj Z[N-k]) / 2
// for the kept columns k = z in [sx0, sx0 + HW) held by this thread
// (u[i] = Z[2 brev(i) + hf]), plus the Nyquist column k = N from Z[0].
// Z[k] and Z[N-k] have the same parity, so both are in this thread; the
// parity is a runtime (warp-uniform) value and selects the partner slot and
// the twiddle, so both parities share this code.
template <int N, int HW>
__device__ __forceinline__ void splitKept(const float2 (&u)[N / 2], int hf, int sx0, float2* crow) {
    constexpr int HALF = N / 2, LOG = ilog2T(HALF);
#pragma unroll
    for (int i = 0; i < HALF; i++) {
        const int z0 = 2 * brevT<LOG>(i);
        const int p0 = brevT<LOG>(((N - z0) & (N - 1)) >> 1);        // partner slot, even parity
        const int p1 = brevT<LOG>(((N - z0 - 1) & (N - 1)) >> 1);    // partner slot, odd parity
        const int z = z0 + hf;
        if ((unsigned)(z - sx0) < (unsigned)HW) {
            const float2 zk = u[i];
            const float2 zm = hf ? u[p1] : u[p0];
            const float2 te = tw128(z0 * (64 / N)), to = tw128((z0 + 1) * (64 / N));  // exp(-2 pi i z / 2N)
            const float tx = hf ? to.x : te.x, ty = hf ? to.y : te.y;
            // even = (zk + conj zm) / 2, odd = -i (zk - conj zm) / 2
            const float ex = 0.5f * (zk.x + zm.x), ey = 0.5f * (zk.y - zm.y);
            const float ox = 0.5f * (zk.y + zm.y), oy = -0.5f * (zk.x - zm.x);
            crow[z - sx0] = make_float2(ex + (tx * ox - ty * oy), ey + (tx * oy + ty * ox));
        }
    }
    if (hf == 0 && (unsigned)(N - sx0) < (unsigned)HW) crow[N - sx0] = make_float2(u[0].x - u[0].y, 0.0f);
}

}  // namespace

// N: packed complex samples per row (W/2), H: FFT-window rows, HW: IFFT
// window size (h = w), NBUF: tile buffers per block.  blockDim.x = 2H.
template <int N, int H, int HW, bool U16, int NBUF>
__global__ void __launch_bounds__(256, 2) k_forward_tma(const __grid_constant__ CUtensorMap tmap, DhFwdParams p) {
    constexpr int HALF = N / 2;
    constexpr int LOGHW = ilog2T(HW);
    constexpr int ES = U16 ? 2 : 4;
    constexpr int ROWB = 2 * N * ES;
    constexpr int NBOX = ROWB / 128;
    constexpr int BOXPX = 128 / ES;
    constexpr int NT = 2 * H;
    constexpr int w = HW, h = HW;
    constexpr int Q = H / HW;
    extern __shared__ unsigned char smRaw[];
    const int P = p.polCount;
    const int tid = threadIdx.x;
    constexpr unsigned tileBytes = (unsigned)H * ROWB;

    // shared layout: tiles (1024-aligned for the swizzle), column buffer
    // [H][w+1], exchange [HW][Q][w], tables, barriers
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smRaw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* tiles = base;
    float2* colbuf = reinterpret_cast<float2*>(tiles + (size_t)NBUF * tileBytes);
    constexpr int CLD = w + 1;
    float2* exch = colbuf + (size_t)H * CLD;
    float2* tCol = exch + (size_t)H * w;            // [P][h][Q]
    float2* tAdj = tCol + (size_t)P * h * Q;         // [P][h][w]
    uint64_t* bars = reinterpret_cast<uint64_t*>(tAdj + (size_t)P * h * w);

    for (int e = tid; e < P * h * Q; e += NT) tCol[e] = p.tabCol[e];
    for (int e = tid; e < P * h * w; e += NT) tAdj[e] = p.tabAdj[e];
    if (tid == 0) {
        for (int b = 0; b < NBUF; b++) mbarInit(&bars[b], 1);
        mbarInitFence();
    }
    __syncthreads();

    const int units = p.frameCount * P;
    const int rowsPerFrame = (int)(p.frameStride / p.frameWidth);
    auto issue = [&](int unit, int buf) {
        const int pol = unit % P, frame = unit / P;
        unsigned char* dst = tiles + (size_t)buf * tileBytes;
        proxyFence();
        mbarExpectTx(&bars[buf], tileBytes);
#pragma unroll
        for (int k = 0; k < NBOX; k++)
            tmaLoad2D(dst + (size_t)k * H * 128, &tmap, p.cx[pol] + k * BOXPX, frame * rowsPerFrame + p.cy[pol], &bars[buf]);
    };
    if (tid == 0 && (int)blockIdx.x < units) issue(blockIdx.x, 0);

    // thread -> (row, parity): warps alternate parity, 32 rows per warp pair
    const int warp = tid >> 5;
    const int hf = warp & 1;
    const int r = (tid & 31) + 32 * (warp >> 1);

    int it = 0;
    for (int unit = blockIdx.x; unit < units; unit += gridDim.x, it++) {
        const int buf = NBUF == 2 ? (it & 1) : 0;
        const unsigned parity = NBUF == 2 ? ((it >> 1) & 1) : (it & 1);
        if (NBUF == 2 && tid == 0 && unit + (int)gridDim.x < units) issue(unit + gridDim.x, buf ^ 1);
        if (!mbarWait(&bars[buf], parity)) {
            if (p.status) {
                *(volatile int*)p.status = 1;
                __threadfence_system();
            }
            // the other buffer may still be filling: wait for it (bounded) before leaving
            if (NBUF == 2 && unit + (int)gridDim.x < units) mbarWait(&bars[buf ^ 1], NBUF == 2 ? (((it + 1) >> 1) & 1) : 0);
            return;
        }
        const int pol = unit % P, frame = unit / P;
        const int sx0 = p.sx0[pol];
        const unsigned char* tile = tiles + (size_t)buf * tileBytes;

        // 1-2. row transforms and the R2C split of the kept columns
        {
            float2 u[HALF];
            float2* crow = colbuf + (size_t)r * CLD;
            if (hf == 0) loadRow<N, 0, U16>(tile, H, r, u);
            else loadRow<N, 1, U16>(tile, H, r, u);
            fftDIF<HALF>(u);
            splitKept<N, HW>(u, hf, sx0, crow);
        }
        __syncthreads();  // column buffer complete; this tile buffer is free
        if (NBUF == 1 && tid == 0 && unit + (int)gridDim.x < units) issue(unit + gridDim.x, 0);

        // 3a. column transforms of the decimated sequences X[Q a + b][c], a < HW
        for (int e = tid; e < w * Q; e += NT) {
            const int c = e % w, b = e / w;
            float2 v[HW];
#pragma unroll
            for (int a = 0; a < HW; a++) v[a] = colbuf[(size_t)(Q * a + b) * CLD + c];
            fftDIF<HW>(v);
#pragma unroll
            for (int i = 0; i < HW; i++) exch[((size_t)brevT<LOGHW>(i) * Q + b) * w + c] = v[i];
        }
        __syncthreads();

        // 3b. kept rows: Y = sum_b tCol[j][b] Z_b[row mod HW], then the window factors
        float2 bc = make_float2(1.0f, 0.0f);
        if (p.batchCal && p.batchCalCount > 0)
            bc = p.batchCal[pol * p.batchCalCount + ((p.frameOffset + frame) % p.batchCalCount)];
        const int sy = p.sy[pol];
        float2* out = p.window + (size_t)(frame * P + pol) * h * w;
        const float2* tc0 = tCol + (size_t)pol * h * Q;
        const float2* ta0 = tAdj + (size_t)pol * h * w;
        for (int e = tid; e < h * w; e += NT) {
            const int j = e / w, c = e - j * w;
            const int row = (j + sy + H / 2) & (H - 1);
            const float2* zb = exch + (size_t)(row & (HW - 1)) * Q * w + c;
            const float2* tc = tc0 + (size_t)j * Q;
            float2 Y = zb[0];
            for (int b = 1; b < Q; b++) Y = cadd(Y, cmul(zb[(size_t)b * w], tc[b]));
            out[e] = cmul(cmul(Y, bc), ta0[e]);
        }
        // the next unit's row stage writes only the column buffer, which no
        // thread reads after the barrier above
    }
}

namespace {

template <int N, int H, int HW, bool U16, int NBUF>
cudaError_t launchTma(const DhFwdParams& p, const CUtensorMap& map, cudaStream_t s) {
    const int ES = U16 ? 2 : 4;
    const size_t tileBytes = (size_t)H * 2 * N * ES;
    const int P = p.polCount, Q = H / HW;
    const size_t smem = 1024 + NBUF * tileBytes +
                        sizeof(float2) * ((size_t)H * (p.w + 1) + (size_t)H * p.w + (size_t)P * p.h * Q + (size_t)P * p.h * p.w) +
                        NBUF * sizeof(uint64_t);
    if (smem > 227 * 1024) return cudaErrorNotSupported;
    auto kern = k_forward_tma<N, H, HW, U16, NBUF>;
    cudaError_t e = setSmemOnce(reinterpret_cast<const void*>(kern), (int)smem);
    if (e != cudaSuccess) return e;
    static int perSM = 0;   // per instantiation; the shared memory and block size are fixed by it
    if (perSM == 0) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, 2 * H, smem);
        if (e != cudaSuccess) return e;
    }
    if (perSM < 1) return cudaErrorNotSupported;
    const int units = p.frameCount * P;
    const int grid = units < perSM * smCountCached() ? units : perSM * smCountCached();
    kern<<<grid, 2 * H, smem, s>>>(map, p);
    return cudaGetLastError();
}

template <int N, bool U16, int NBUF>
cudaError_t dispatchH(const DhFwdParams& p, const CUtensorMap& map, cudaStream_t s) {
    const int H = 1 << p.logH;
    if (p.h == 16) {
        if (H == 128) return launchTma<N, 128, 16, U16, NBUF>(p, map, s);
        if (H == 64) return launchTma<N, 64, 16, U16, NBUF>(p, map, s);
        if (H == 32) return launchTma<N, 32, 16, U16, NBUF>(p, map, s);
    } else if (p.h == 32) {
        if (H == 128) return launchTma<N, 128, 32, U16, NBUF>(p, map, s);
        if (H == 64) return launchTma<N, 64, 32, U16, NBUF>(p, map, s);
        if (H == 32) return launchTma<N, 32, 32, U16, NBUF>(p, map, s);
    }
    return cudaErrorNotSupported;
}

cudaError_t dispatchTma(const DhFwdParams& p, const CUtensorMap& map, cudaStream_t s) {
    const int W = 1 << p.logW;
    if (p.inputU16) {
        if (W == 128) return dispatchH<64, true, 2>(p, map, s);
        if (W == 64) return dispatchH<32, true, 2>(p, map, s);
    } else {
        if (W == 128) return dispatchH<64, false, 1>(p, map, s);
        if (W == 64) return dispatchH<32, false, 2>(p, map, s);
        if (W == 32) return dispatchH<16, false, 2>(p, map, s);
    }
    return cudaErrorNotSupported;
}

}  // namespace

// Returns cudaErrorNotSupported when the shape, the alignment or the driver
// rules this kernel out (the caller then uses k_forward_reg / k_forward).
cudaError_t dh_launch_forward_tma(const DhFwdParams& p, cudaStream_t s) {
    const int W = 1 << p.logW, H = 1 << p.logH;
    const int es = p.inputU16 ? 2 : 4;
    if (p.frameCount <= 0) return cudaSuccess;
    if (!p.tabCol || !p.tabAdj) return cudaErrorNotSupported;
    if (p.h != p.w || (p.h != 16 && p.h != 32) || H < 32 || H > 128 || H < p.h) return cudaErrorNotSupported;
    if (W * es < 128 || W > 128) return cudaErrorNotSupported;
    const int N = W / 2;
    for (int q = 0; q < p.polCount; q++) {
        if (p.sx0[q] < 0 || p.sx0[q] + p.w > N + 1) return cudaErrorNotSupported;
        if ((p.cx[q] * es) % 16 != 0) return cudaErrorNotSupported;   // TMA x coordinate: 16-byte multiple
    }
    if ((reinterpret_cast<uintptr_t>(p.frames) % 16) != 0 || ((size_t)p.frameWidth * es) % 16 != 0) return cudaErrorNotSupported;
    if (p.frameStride % p.frameWidth != 0) return cudaErrorNotSupported;
    const long long rowsPerFrame = p.frameStride / p.frameWidth;
    const long long totalRows = rowsPerFrame * p.frameCount;
    if (totalRows >= (1ll << 31)) return cudaErrorNotSupported;
    CUtensorMap map;
    if (!frameTensorMap(map, p.frames, p.inputU16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, es,
                        (unsigned long long)p.frameWidth, (unsigned long long)totalRows, (unsigned)(128 / es), (unsigned)H))
        return cudaErrorNotSupported;

    return dispatchTma(p, map, s);
}
