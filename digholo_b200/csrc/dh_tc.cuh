// tcgen05 / mbarrier / bulk-copy helpers shared by the tensor-core overlap
// kernels: inline PTX for sm_100a (5th-generation tensor cores, tensor
// memory), the K-major 128-byte-swizzled shared-memory operand layout and
// the exact split of int16 values into bf16 hi + lo.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dh {
namespace tc {

__device__ __forceinline__ uint32_t sAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInitTc(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sAddr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbarWaitTc(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(sAddr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);          // start address
    d |= (uint64_t)(16 >> 4) << 16;                   // leading byte offset (unused with this swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;                 // stride byte offset
    d |= (uint64_t)1 << 46;                           // version
    d |= (uint64_t)2 << 61;                           // 128-byte swizzle
    return d;
}

// Instruction descriptor, kind::f16: bf16 A and B, FP32 accumulator, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t instrDesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mmaBf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mmaCommit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sAddr(bar))
                 : "memory");
}
__device__ __forceinline__ void mbarExpectTxTc(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sAddr(bar)), "r"(bytes) : "memory");
}
// One contiguous global -> shared copy (16-byte aligned addresses, size a
// multiple of 16) completing on `bar`.
__device__ __forceinline__ void bulkLoad(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sAddr(dst)),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(sAddr(bar))
                 : "memory");
}
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive accumulator columns of this warp's 32 lanes.
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Exact split of 8 int16 values into bf16 hi and lo (element order kept).
__device__ __forceinline__ void split8(const uint4 raw, uint4& hi, uint4& lo) {
    const unsigned w[4] = {raw.x, raw.y, raw.z, raw.w};
    unsigned h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float a = (float)(short)(w[i] & 0xFFFFu);
        const float b = (float)(short)(w[i] >> 16);
        const __nv_bfloat162 hb = __floats2bfloat162_rn(a, b);
        const __nv_bfloat162 lb = __floats2bfloat162_rn(a - __low2float(hb), b - __high2float(hb));
        h[i] = *reinterpret_cast<const unsigned*>(&hb);
        l[i] = *reinterpret_cast<const unsigned*>(&lb);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Byte offset of 16-byte chunk q (elements 8q .. 8q+7 along K) of row r in a
// K-major 128-byte-swizzled operand with `rows` rows: 64-element atoms of
// rows x 128 bytes, chunk c of row r stored at chunk c ^ (r & 7).
__device__ __forceinline__ uint32_t swzOffset(int rows, int r, int q) {
    const int atom = q >> 3, c = q & 7;
    return (uint32_t)(atom * rows * 128 + r * 128 + ((c ^ (r & 7)) << 4));
}

}  // namespace tc
}  // namespace dh
