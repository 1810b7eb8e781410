// digHoloB200ProcessBatchNoAlloc: the batch path for callers that cannot
// allocate device memory at the time they process frames -- for example a
// real-time acquisition callback that must not block in cudaMalloc/cudaFree
// (both can synchronise the device), or code running under an allocator
// policy that forbids new allocations after start-up.
//
// The forward kernel hands the Fourier windows to the inverse kernel through
// a scratch buffer.  Here that scratch is a file-scope static device array of
// fixed size instead of a handle-owned allocation, and the caller passes the
// frames and every output buffer.  Nothing in this entry point allocates.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "dh_object.h"

// Scratch for the Fourier windows [frame][pol][h][w] of one call: 8 MiB.
// Every GPU that loads this library holds it until the process exits.
#define DH_NOALLOC_WINDOW_BYTES (8u << 20)
static __device__ __align__(256) float2 g_noallocWindow[DH_NOALLOC_WINDOW_BYTES / sizeof(float2)];

dh::Object* dhObjectForHandle(int handleIdx);

namespace dh {
int objProcessNoAlloc(Object& o, const void* frames, int frameCount, int u16, float2* window, size_t windowBytes,
                      float2* coefs, short* fieldR, short* fieldI, float* stats);
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex gSetupLock;
void* gScratch[kMaxDevices] = {nullptr};
}  // namespace

extern "C" {

typedef float complex64[2];

// Processes `frameCount` frames already in device memory with the
// configuration of `handleIdx`, writing into caller-owned device buffers:
//   coefs  [frame][pol * modeCount]          complex64 (may be null when maxMG = 0)
//   fieldR, fieldI [frame][pol][ny][nx]      int16
//   stats  [7][pol][frameCount + 1]          float (DIGHOLO_ANALYSIS layout; the
//                                            last column, the batch aggregate, is not written)
// The handle must already hold the tables for this configuration: process one
// batch with digHoloProcessBatch or digHoloB200ProcessBatchDevice first (that
// call allocates).  frameCount * polCount * w * h * 8 bytes must not exceed
// the 8 MiB scratch (e.g. 2048 dual-polarisation frames with 16x16 IFFT
// windows), and frameCount must not exceed the batch that call prepared
// where that batch sized a scratch of the handle (the Fourier planes of
// 256-pixel and wider windows, the band buffers of large full-resolution
// fields): larger calls return DIGHOLO_ERROR_MEMORYALLOCATION instead of
// allocating.  The call makes the handle's device current (and leaves it
// current); the first call on a device then looks up the scratch address on
// that device with cudaGetSymbolAddress (with CUDA's lazy module loading that
// lookup is also when the 8 MiB array is placed in device memory), so make
// that first call before any stream capture.  All calls share the one scratch array and it keeps the
// last call's contents (the forward kernel overwrites every element it reads
// back, so nothing needs clearing); calls whose GPU work overlaps race on it.
int digHoloB200ProcessBatchNoAlloc(int handleIdx, const void* frames, int frameCount, int framesAreUint16,
                                   complex64* coefs, short* fieldR, short* fieldI, float* stats) {
    dh::Object* o = dhObjectForHandle(handleIdx);
    if (!o) return dh::ERR_INVALIDHANDLE;
    if (!frames || !fieldR || !fieldI || !stats) return dh::ERR_NULLPOINTER;
    if (frameCount < 1) return dh::ERR_INVALIDDIMENSION;
    // the handle's device (set by its first batch; calls on one handle are
    // serialised by the caller): the scratch address is looked up and cached
    // on that device, whichever device the calling thread had current
    const int dev = o->device;
    void* scratch = nullptr;
    if (dev >= kMaxDevices) return dh::ERR_ERROR;
    if (dev >= 0) {
        cudaError_t e = cudaSetDevice(dev);
        if (e != cudaSuccess) return dh::ERR_ERROR;
        std::lock_guard<std::mutex> g(gSetupLock);
        if (!gScratch[dev]) {
            // the array's name is a host-side stand-in; the kernels need its device address
            e = cudaGetSymbolAddress(&gScratch[dev], g_noallocWindow);
            if (e != cudaSuccess) {
                gScratch[dev] = nullptr;
                fprintf(stderr, "digholo_b200: cudaGetSymbolAddress for the no-alloc scratch failed: %s\n",
                        cudaGetErrorString(e));
                return dh::ERR_ERROR;
            }
        }
        scratch = gScratch[dev];
    }
    // an unprepared handle (no device yet, scratch null) is refused there
    return dh::objProcessNoAlloc(*o, frames, frameCount, framesAreUint16 ? 1 : 0, static_cast<float2*>(scratch),
                                 DH_NOALLOC_WINDOW_BYTES, reinterpret_cast<float2*>(coefs), fieldR, fieldI, stats);
}

}  // extern "C"
