// Auxiliary entry points of the digHolo interface around the batch path:
// frame buffers and batch calibrations from files, the basis fields, the
// console redirection, configuration backups, the Zernike coefficient rows,
// the thread-count estimate and the debug hook; and the viewport entry
// points, whose bitmap renderer is not part of this library (they return
// nothing and say so).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <vector>

#include "dh_object.h"
#include "dh_sim.h"

using dh::Object;

dh::Object* dhObjectForHandle(int h);

namespace dh {

FILE* gConsole = nullptr;   // digHoloConsoleRedirectToFile; stdout when null
FILE* console() { return gConsole ? gConsole : stdout; }

// Basis fields of the handle's current basis on its reconstructed plane
// (GetFieldsBasis, digHolo.cpp:5233-5305): output mode j of polarisation p
// is sum_i T[i][j] HG_i (T the identity for HG, the [in][out] matrix for a
// custom basis, the LG transform for LG), formed as generateModeSeparable
// forms it, [mode][pol][ny][nx] complex, into o.hBasisFields.
int objBasisFields(Object& o, int* modeCountOut) {
    std::lock_guard<std::mutex> guard(o.lock);
    const int M = o.modeCount, P = o.polCount, G = o.cfg.maxMG;
    if (M <= 0 || G <= 0 || !o.dHgX.ptr || !o.dHgY.ptr) return ERR_NULLPOINTER;
    const int nx = o.geo.nx, ny = o.geo.ny;
    // transform columns: the active output basis of the last batch
    int dout = M, din = M;
    std::vector<float2> T;
    if (o.basisActive != 0 && o.dBasisT.ptr) {
        din = o.basisDimIn;
        dout = o.modeCountOut;
        T.resize((size_t)din * dout);
        DH_CUDA(o, cudaMemcpy(T.data(), o.dBasisT.ptr, T.size() * sizeof(float2), cudaMemcpyDeviceToHost));
    }
    std::vector<float> sx((size_t)P * G), sy((size_t)P * G);
    DH_CUDA(o, cudaMemcpy(sx.data(), o.dHgScaleX.ptr, sx.size() * 4, cudaMemcpyDeviceToHost));
    DH_CUDA(o, cudaMemcpy(sy.data(), o.dHgScaleY.ptr, sy.size() * 4, cudaMemcpyDeviceToHost));
    std::vector<int> mIdx(M), nIdx(M);
    for (int g = 0, k = 0; g < G && k < M; g++)
        for (int q = 0; q <= g && k < M; q++, k++) { mIdx[k] = g - q; nIdx[k] = q; }
    std::vector<DhSimMode> terms;
    std::vector<int> offs((size_t)dout * P + 1, 0);
    int maxTerms = 1;
    for (int j = 0; j < dout; j++) {
        for (int p = 0; p < P; p++) {
            const size_t u = (size_t)j * P + p;
            offs[u] = (int)terms.size();
            for (int k = 0; k < M; k++) {
                float cr = 0.f, ci = 0.f;
                if (T.empty()) {
                    cr = (k == j) ? 1.f : 0.f;
                } else if (k < din) {
                    cr = T[(size_t)k * dout + j].x;
                    ci = T[(size_t)k * dout + j].y;
                }
                const double xs = sx[(size_t)p * G + mIdx[k]], ys = sy[(size_t)p * G + nIdx[k]];
                const float cR = (float)(xs * ys * cr), cI = (float)(xs * ys * ci);
                const float pw = cR * cR + cI * cI;
                if (pw > 0 || k == 0 || k == M - 1) terms.push_back({cR, cI, mIdx[k], nIdx[k]});
            }
            maxTerms = std::max(maxTerms, (int)terms.size() - offs[u]);
        }
    }
    offs[(size_t)dout * P] = (int)terms.size();
    DevBuf dTerms, dOffs, dOut;
    DH_CUDA(o, dTerms.ensure(terms.size() * sizeof(DhSimMode)));
    DH_CUDA(o, dOffs.ensure(offs.size() * sizeof(int)));
    const size_t n = (size_t)dout * P * nx * ny;
    DH_CUDA(o, dOut.ensure(n * sizeof(float2)));
    DH_CUDA(o, cudaMemcpyAsync(dTerms.ptr, terms.data(), terms.size() * sizeof(DhSimMode), cudaMemcpyHostToDevice, o.stream));
    DH_CUDA(o, cudaMemcpyAsync(dOffs.ptr, offs.data(), offs.size() * sizeof(int), cudaMemcpyHostToDevice, o.stream));
    DhSimFieldArgs a;
    memset(&a, 0, sizeof(a));
    a.modes = dTerms.as<DhSimMode>();
    a.modeOffset = dOffs.as<int>();
    a.hgCol = o.dHgX.as<short>();
    a.hgRow = o.dHgY.as<short>();
    a.frames = dout;
    a.polCount = P;
    a.rows = ny;
    a.cols = nx;
    a.frameWidth = nx;
    a.G = G;
    DH_CUDA(o, dh_launch_basis_fields(a, maxTerms, dOut.as<float2>(), o.stream));
    if (!o.hBasisFields.ensure(n * sizeof(float2))) return fail(o, ERR_MEMORYALLOCATION, "host basis field buffer");
    DH_CUDA(o, cudaMemcpyAsync(o.hBasisFields.ptr, dOut.ptr, n * sizeof(float2), cudaMemcpyDeviceToHost, o.stream));
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    *modeCountOut = dout;
    return ERR_SUCCESS;
}

}  // namespace dh

extern "C" {

typedef float complex64[2];

// digHolo.h:288 / digHolo.cpp:4274-4350: uint16 frames from a binary file,
// held by the handle as float32 and set as its frame buffer.
int digHoloSetFrameBufferFromFile(int h, const char* fname) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    if (!fname) return dh::ERR_NULLPOINTER;
    std::ifstream f(fname, std::ios::binary);
    if (!f) {
        fprintf(dh::console(), "FrameBuffer file could not be opened. %s\n", fname);
        fflush(dh::console());
        return 11;   // DIGHOLO_ERROR_FILENOTFOUND
    }
    f.seekg(0, std::ios::end);
    const size_t bytes = (size_t)f.tellg();
    f.seekg(0, std::ios::beg);
    if (bytes % 2) return dh::ERR_INVALIDDIMENSION;
    std::vector<unsigned short> raw(bytes / 2);
    f.read(reinterpret_cast<char*>(raw.data()), (std::streamsize)bytes);
    std::lock_guard<std::mutex> g(o->lock);
    o->ownFrames.assign(raw.begin(), raw.end());
    o->frames = o->ownFrames.data();
    o->framesU16 = 0;
    o->framesTransposed = 0;
    o->framesOnDevice = 0;
    return dh::ERR_SUCCESS;
}

// digHolo.h:624 / digHolo.cpp:4536-4590: polCount x batchCount complex64.
int digHoloConfigSetBatchCalibration(int h, complex64* cal, int polCount, int batchCount);
int digHoloConfigSetBatchCalibrationEnabled(int h, int enabled);
int digHoloConfigSetBatchCalibrationFromFile(int h, const char* fname, int polCount, int batchCount) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    std::ifstream f(fname ? fname : "", std::ios::binary);
    if (!fname || !f) {
        digHoloConfigSetBatchCalibrationEnabled(h, 0);
        return 11;   // DIGHOLO_ERROR_FILENOTFOUND
    }
    f.seekg(0, std::ios::end);
    const size_t bytes = (size_t)f.tellg();
    f.seekg(0, std::ios::beg);
    if (polCount <= 0 || batchCount <= 0 || bytes != (size_t)polCount * batchCount * sizeof(complex64)) {
        digHoloConfigSetBatchCalibrationEnabled(h, 0);
        return dh::ERR_INVALIDDIMENSION;
    }
    std::vector<float> cal(bytes / 4);
    f.read(reinterpret_cast<char*>(cal.data()), (std::streamsize)bytes);
    return digHoloConfigSetBatchCalibration(h, reinterpret_cast<complex64*>(cal.data()), polCount, batchCount);
}

// digHolo.h:1587 / digHolo.cpp:15378 and 5233-5305
complex64* digHoloBasisGetFields(int h, int* modeCount, int* polCount, float** x, float** y, int* width, int* height) {
    Object* o = dhObjectForHandle(h);
    int m = 0;
    if (!o || !o->processedOverlap || dh::objBasisFields(*o, &m) != dh::ERR_SUCCESS) {
        *modeCount = 0; *polCount = 0; *x = nullptr; *y = nullptr; *width = 0; *height = 0;
        return nullptr;
    }
    o->hX = o->geo.x;
    o->hY = o->geo.y;
    *modeCount = m;
    *polCount = o->polCount;
    *x = o->hX.data();
    *y = o->hY.data();
    *width = o->geo.nx;
    *height = o->geo.ny;
    return static_cast<complex64*>(o->hBasisFields.ptr);
}

// digHolo.h:1766 / digHolo.cpp:15312: the reference times its CPU thread
// pool; the GPU path has no thread count to tune, so the configured count
// is returned.
int digHoloBenchmarkEstimateThreadCountOptimal(int h, float goalDuration) {
    (void)goalDuration;
    Object* o = dhObjectForHandle(h);
    return o ? o->cfg.threadCount : 0;
}

// digHolo.h:1883-1897 / digHolo.cpp:15578-15640.  The viewport renders
// frames, Fourier planes and fields into RGB bitmaps for display; that
// renderer is not part of this library.  No bitmap, width = height = 0.
unsigned char* digHoloGetViewport(int h, int displayMode, int waitForNewFrame, int* width, int* height,
                                  char** windowString) {
    (void)h; (void)displayMode; (void)waitForNewFrame;
    static char msg[] = "digholo_b200: the viewport is not available in this library";
    if (width) *width = 0;
    if (height) *height = 0;
    if (windowString) *windowString = msg;
    return nullptr;
}
int digHoloGetViewportToFile(int h, int displayMode, int forceProcessing, int* width, int* height,
                             char** windowString, const char* filename) {
    (void)filename;
    if (!dhObjectForHandle(h)) return dh::ERR_INVALIDHANDLE;
    digHoloGetViewport(h, displayMode, forceProcessing, width, height, windowString);
    return dh::ERR_ERROR;
}

// digHolo.h:1945-1952 / digHolo.cpp:15641-15684: library messages to a
// file, and back to stdout.
int digHoloConsoleRestore() {
    if (dh::gConsole && dh::gConsole != stdout) fclose(dh::gConsole);
    dh::gConsole = nullptr;
    return dh::ERR_SUCCESS;
}
int digHoloConsoleRedirectToFile(char* filename) {
    if (!filename) {
        digHoloConsoleRestore();
        return dh::ERR_NULLPOINTER;
    }
    FILE* f = fopen(filename, "w");
    if (!f) {
        digHoloConsoleRestore();
        return 10;   // DIGHOLO_ERROR_FILENOTCREATED
    }
    if (dh::gConsole && dh::gConsole != stdout) fclose(dh::gConsole);
    dh::gConsole = f;
    return dh::ERR_SUCCESS;
}

// digHolo.h:1973-1983 / digHolo.cpp:13103-13140
int digHoloConfigBackupSave(int h) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    o->cfgBackup = o->cfg;
    o->cfgBackupValid = 1;
    return dh::ERR_SUCCESS;
}
// Before any save the backup holds the configuration a handle starts with.
int digHoloConfigBackupLoad(int h) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    o->cfg = o->cfgBackup;
    return dh::ERR_SUCCESS;
}

// digHolo.h:1990 (not for general use): nothing to run here.
void digHoloDebugRoutine(int h) { (void)h; }

// digHolo.h:2075-2084 / digHolo.cpp:14203-14216: the per-polarisation rows of Zernike
// coefficients (piston, tilt x, tilt y, ..., defocus at index 4; six per row).
float** digHoloConfigGetZernCoefs(int h) {
    Object* o = dhObjectForHandle(h);
    if (!o) return nullptr;
    for (int p = 0; p < dh::POLMAX; p++) o->zernRows[p] = o->cfg.zern[p];
    return o->zernRows;
}
int digHoloConfigGetZernCount(int h) { return dhObjectForHandle(h) ? 6 : 0; }

}  // extern "C"

// ------------------------------------------------------------ wavelengths
// digHolo.h:832 / digHolo.cpp:14611 and 6658-6684: the array takes effect
// at the next processing (or GetWavelengths).
extern "C" int digHoloConfigSetWavelengths(int h, float* wavelengths, int wavelengthCount) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    if (wavelengthCount <= 0) return dh::ERR_INVALIDARGUMENT;
    if (!wavelengths) return dh::ERR_NULLPOINTER;
    std::lock_guard<std::mutex> g(o->lock);
    o->wavelengthsNew.assign(wavelengths, wavelengths + wavelengthCount);
    o->wavelengthsValid = 0;
    return dh::ERR_SUCCESS;
}

// digHolo.h:843 / digHolo.cpp:14644 and 6578-6656: wavelengths equally
// spaced in frequency, lambda_i = c0 / (c0 / start + i df), df = (c0 / stop
// - c0 / start) / (count - 1), in float32 with c0 the integer 299792458.
// A single step keeps the reference's choices, including its use of half
// the start wavelength when the stop wavelength is invalid.
static int linearFrequency(Object& o, float lambdaStart, float lambdaStop, int lambdaCount) {
    if (lambdaCount <= 0) return dh::ERR_INVALIDDIMENSION;
    const int c0 = 299792458;
    float fStart = c0 / lambdaStart;
    const float fStop = c0 / lambdaStop;
    float df = (fStop - fStart) / (lambdaCount - 1);
    if (lambdaCount <= 1) {
        if (lambdaStop <= 0 && lambdaStart > 0) {
            fStart = c0 / (lambdaStart / 2);
        } else if (lambdaStart <= 0 && lambdaStop > 0) {
            fStart = c0 / (lambdaStart / 2);
        } else if (lambdaStart <= 0 && lambdaStop <= 0) {
            fStart = c0 / o.cfg.wavelengthCentre;
        } else {
            fStart = c0 / ((lambdaStop + lambdaStart) / 2);
        }
        df = 0;
    }
    std::vector<float> w(lambdaCount);
    for (int i = 0; i < lambdaCount; i++) {
        const float f0 = fStart + df * i;
        w[i] = c0 / f0;
    }
    o.wavelengthsNew = w;
    o.wavelengthsValid = 0;
    return dh::ERR_SUCCESS;
}

extern "C" int digHoloConfigSetWavelengthsLinearFrequency(int h, float wavelengthStart, float wavelengthStop,
                                                          int wavelengthCount) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    if (!wavelengthCount) return dh::ERR_INVALIDARGUMENT;
    std::lock_guard<std::mutex> g(o->lock);
    return linearFrequency(*o, wavelengthStart, wavelengthStop, wavelengthCount);
}

// digHolo.h:854 / digHolo.cpp:14630 and 5056-5068
extern "C" float* digHoloConfigGetWavelengths(int h, int* wavelengthCount) {
    Object* o = dhObjectForHandle(h);
    if (!o) return nullptr;
    std::lock_guard<std::mutex> g(o->lock);
    if (o->wavelengths.empty()) {   // nothing processed yet: no array in use
        *wavelengthCount = 0;
        return nullptr;
    }
    dh::objWavelengthUpdate(*o);
    *wavelengthCount = (int)o->wavelengths.size();
    return o->wavelengths.data();
}

// digHolo.h:886-895 / digHolo.cpp:14662-14698
extern "C" int digHoloConfigSetWavelengthOrdering(int h, int inoutIdx, int ordering) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    if ((inoutIdx == 0 || inoutIdx == 1) && (ordering == 0 || ordering == 1)) {
        o->cfg.wavelengthOrdering[inoutIdx] = ordering;
        return dh::ERR_SUCCESS;
    }
    return dh::ERR_INVALIDARGUMENT;
}
extern "C" int digHoloConfigGetWavelengthOrdering(int h, int inoutIdx) {
    Object* o = dhObjectForHandle(h);
    if (!o) return 0;
    return (inoutIdx == 0 || inoutIdx == 1) ? o->cfg.wavelengthOrdering[inoutIdx] : 0;
}

extern "C" complex64* digHoloProcessBatch(int h, int* batchCount, int* modeCount, int* polCount);

// digHolo.h:1510 / digHolo.cpp:15194 and 5046-5054
extern "C" complex64* digHoloProcessBatchFrequencySweepLinear(int h, int* batchCount, int* modeCount, int* polCount,
                                                              float lambdaStart, float lambdaStop, int lambdaCount) {
    Object* o = dhObjectForHandle(h);
    if (!o) {
        *batchCount = 0; *modeCount = 0; *polCount = 0;
        return nullptr;
    }
    {
        std::lock_guard<std::mutex> g(o->lock);
        linearFrequency(*o, lambdaStart, lambdaStop, lambdaCount);
    }
    return digHoloProcessBatch(h, batchCount, modeCount, polCount);
}

// digHolo.h:1525 / digHolo.cpp:15217 and 5070-5078
extern "C" complex64* digHoloProcessBatchWavelengthSweepArbitrary(int h, int* batchCount, int* modeCount, int* polCount,
                                                                  float* wavelengths, int lambdaCount) {
    Object* o = dhObjectForHandle(h);
    if (!o) {
        *batchCount = 0; *modeCount = 0; *polCount = 0;
        return nullptr;
    }
    if (lambdaCount > 0 && wavelengths) {
        std::lock_guard<std::mutex> g(o->lock);
        o->wavelengthsNew.assign(wavelengths, wavelengths + lambdaCount);
        o->wavelengthsValid = 0;
    }
    return digHoloProcessBatch(h, batchCount, modeCount, polCount);
}

// ------------------------------------------------------------ reference-wave calibration
// digHolo.h:369-437 / digHolo.cpp:5309-5540.  The factors are stored as the
// reference forms them: from an intensity, sqrt(1 / (I / max I)); from a
// field, the componentwise (1 / (re / max|E|), -1 / (im / max|E|)); NaN or
// infinite factors become 0.  Their reconstructed planes multiply the IFFT
// output of each frame of the calibration's size (dh_refcal.cpp).
namespace {
int refCalStore(Object& o, const unsigned short* i16, const float* c64, int count, int w, int h) {
    if (!i16 && !c64) { o.refCalEnabled = 0; return dh::ERR_NULLPOINTER; }
    if (w <= 0 || h <= 0 || count <= 0) { o.refCalEnabled = 0; return dh::ERR_INVALIDARGUMENT; }
    const size_t n = (size_t)w * h * count;
    o.refCal.assign(2 * n, 0.f);
    if (i16) {
        int maxV = 0;
        for (size_t i = 0; i < n; i++) maxV = std::max(maxV, (int)i16[i]);
        const float maxScale = 1.0f / maxV;
        for (size_t i = 0; i < n; i++) {
            float v = 1.0f / ((float)i16[i] * maxScale);
            if (std::isnan(v) || std::isinf(v)) v = 0;
            o.refCal[2 * i] = sqrtf(v);
        }
    } else {
        float maxV = 0;
        for (size_t i = 0; i < n; i++) {
            const float vR = c64[2 * i], vI = c64[2 * i + 1];
            const float v2 = vR * vR + vI * vI;
            if (v2 > maxV) maxV = v2;
        }
        maxV = sqrtf(maxV);
        const float maxScale = 1.0f / maxV;
        for (size_t i = 0; i < n; i++) {
            float vR = 1.0f / (c64[2 * i] * maxScale);
            float vI = -1.0f / (c64[2 * i + 1] * maxScale);
            if (std::isnan(vR) || std::isinf(vR) || std::isnan(vI) || std::isinf(vI)) { vR = 0; vI = 0; }
            o.refCal[2 * i] = vR;
            o.refCal[2 * i + 1] = vI;
        }
    }
    o.refCalWidth = w;
    o.refCalHeight = h;
    o.refCalCount = count;
    o.refCalEnabled = 1;
    o.refCalGen++;
    if (o.device >= 0) cudaSetDevice(o.device);
    o.refCalPlanes.clear();   // frees device planes (cudaFree waits for kernels using them)
    return dh::ERR_SUCCESS;
}
}  // namespace

extern "C" int digHoloConfigSetRefCalibrationIntensity(int h, unsigned short* cal, int wavelengthCount, int width,
                                                       int height) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    std::lock_guard<std::mutex> g(o->lock);
    return refCalStore(*o, cal, nullptr, wavelengthCount, width, height);
}
extern "C" int digHoloConfigSetRefCalibrationField(int h, complex64* cal, int wavelengthCount, int width, int height) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    std::lock_guard<std::mutex> g(o->lock);
    return refCalStore(*o, nullptr, cal ? &cal[0][0] : nullptr, wavelengthCount, width, height);
}
// The file holds uint16 intensities or complex64 fields, told apart by its
// size (digHolo.cpp:5320-5407).
extern "C" int digHoloConfigSetRefCalibrationFromFile(int h, const char* fname, int wavelengthCount, int width,
                                                      int height) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    std::ifstream f(fname ? fname : "", std::ios::binary);
    if (!fname || !f) { o->refCalEnabled = 0; return 11; }   // DIGHOLO_ERROR_FILENOTFOUND
    f.seekg(0, std::ios::end);
    const size_t bytes = (size_t)f.tellg();
    f.seekg(0, std::ios::beg);
    const size_t frame16 = (size_t)width * height * 2, frame32 = (size_t)width * height * 8;
    size_t total16 = frame16 * wavelengthCount, total32 = frame32 * wavelengthCount;
    int count = wavelengthCount;
    if (bytes == frame16) {
        count = 1;
        total16 = frame16;
    } else if (bytes == frame32 && wavelengthCount != 2) {
        count = 1;
        total32 = frame32;
    }
    std::lock_guard<std::mutex> g(o->lock);
    if (bytes == total16) {
        std::vector<unsigned short> v(bytes / 2);
        f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)bytes);
        return refCalStore(*o, v.data(), nullptr, count, width, height);
    }
    if (bytes == total32) {
        std::vector<float> v(bytes / 4);
        f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)bytes);
        return refCalStore(*o, nullptr, v.data(), count, width, height);
    }
    o->refCalEnabled = 0;
    return dh::ERR_INVALIDDIMENSION;
}
extern "C" int digHoloConfigSetRefCalibrationEnabled(int h, int enabled) {
    Object* o = dhObjectForHandle(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    o->refCalEnabled = enabled;
    return dh::ERR_SUCCESS;
}
extern "C" int digHoloConfigGetRefCalibrationEnabled(int h) {
    Object* o = dhObjectForHandle(h);
    return o ? o->refCalEnabled : 0;
}
// The calibration as applied to the reconstructed fields (digHolo.cpp:4912-4924):
// [item][pol][height][width] with the field's axes, for the geometry of the
// last batch; null until a batch with an applicable calibration ran.
extern "C" complex64* digHoloConfigGetRefCalibrationFields(int h, int* wavelengthCount, int* polCount, float** x,
                                                           float** y, int* width, int* height) {
    if (wavelengthCount) *wavelengthCount = 0;
    if (polCount) *polCount = 0;
    if (x) *x = nullptr;
    if (y) *y = nullptr;
    if (width) *width = 0;
    if (height) *height = 0;
    Object* o = dhObjectForHandle(h);
    if (!o) return nullptr;
    std::lock_guard<std::mutex> g(o->lock);
    if (dh::objRefCalFieldsToHost(*o) != dh::ERR_SUCCESS) return nullptr;
    if (wavelengthCount) *wavelengthCount = o->refCalCount;
    if (polCount) *polCount = o->polCount;
    if (x) *x = o->hRefCalX.data();
    if (y) *y = o->hRefCalY.data();
    if (width) *width = o->geo.nx;
    if (height) *height = o->geo.ny;
    return reinterpret_cast<complex64*>(o->hRefCalFields.ptr);
}
