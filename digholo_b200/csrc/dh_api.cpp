// C ABI of digholo_b200: the digHolo entry points of the batch path, with
// the reference's argument meaning, clamping and error returns
// (digHolo.h:209-1776; wrappers digHolo.cpp:13412-15705), plus the
// digHoloB200* extensions for device-resident use.  All names are
// extern "C"; declarations are in include/digHolo.h.
#include <cuda_runtime.h>

#include <cmath>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "dh_object.h"

using dh::Object;

void dh_eigen_destroy(DhEigen* e);

typedef float complex64[2];

namespace {

std::mutex gTableLock;
std::vector<Object*> gObjects;  // index = handle; nullptr once destroyed

Object* get(int h) {
    std::lock_guard<std::mutex> g(gTableLock);
    if (h < 0 || h >= (int)gObjects.size()) return nullptr;
    return gObjects[h];
}

}  // namespace

#define OBJ_OR(h, ret) Object* o = get(h); if (!o) return ret

dh::Object* dhObjectForHandle(int h) { return get(h); }

// Handles created so far (destroyed ones included), for the settings-file
// runner, which uses handle 0 when one exists (digHolo.cpp:16774-16782).
extern "C" int dhHandleCount() {
    std::lock_guard<std::mutex> g(gTableLock);
    return (int)gObjects.size();
}

extern "C" {

// ------------------------------------------------------------ handles
// digHolo.h:209 / digHolo.cpp:13434
int digHoloCreate() {
    Object* o = new Object();
    o->cfg.threadCount = (int)std::thread::hardware_concurrency();
    o->cfgBackup = o->cfg;
    std::lock_guard<std::mutex> g(gTableLock);
    gObjects.push_back(o);
    return (int)gObjects.size() - 1;
}

// digHolo.h:216 / digHolo.cpp:13449 (returns 0 on success, 1 for an unknown handle)
int digHoloDestroy(int h) {
    Object* o = nullptr;
    {
        std::lock_guard<std::mutex> g(gTableLock);
        if (h < 0 || h >= (int)gObjects.size()) return 1;
        o = gObjects[h];
        gObjects[h] = nullptr;
    }
    if (o) {
        if (o->device >= 0) {
            cudaSetDevice(o->device);
            if (o->stream) cudaStreamSynchronize(o->stream);
            dh::objReleaseGraphs(*o);
            if (o->stream && !o->userStream) cudaStreamDestroy(o->stream);
            for (auto e : o->evStage) if (e) cudaEventDestroy(e);
            if (o->copyStream) cudaStreamDestroy(o->copyStream);
            for (auto e : o->evCopy) if (e) cudaEventDestroy(e);
            if (o->copyStream2) cudaStreamDestroy(o->copyStream2);
            for (auto e : o->evCopy2) if (e) cudaEventDestroy(e);
            if (o->d2hStream) cudaStreamDestroy(o->d2hStream);
            for (auto e : o->evChunk) if (e) cudaEventDestroy(e);
            if (o->evD2H) cudaEventDestroy(o->evD2H);
            if (o->evStart) cudaEventDestroy(o->evStart);
            if (o->evStop) cudaEventDestroy(o->evStop);
            if (o->hStatus) cudaFreeHost(o->hStatus);
            if (o->evUpload) cudaEventDestroy(o->evUpload);
            dh_eigen_destroy(o->eigen);
        }
        delete o;
    }
    return 0;
}

// ------------------------------------------------------------ frame source
// digHolo.h:245 / digHolo.cpp:4268
int digHoloSetFrameBuffer(int h, float* buffer) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!buffer) return dh::ERR_NULLPOINTER;
    o->frames = buffer; o->framesU16 = 0; o->framesTransposed = 0; o->framesOnDevice = 0;
    return dh::ERR_SUCCESS;
}
float* digHoloGetFrameBuffer(int h) {
    OBJ_OR(h, nullptr);
    return o->framesU16 ? nullptr : (float*)o->frames;
}
// digHolo.h:268 / digHolo.cpp:4284
int digHoloSetFrameBufferUint16(int h, unsigned short* buffer, int transposeMode) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!buffer) return dh::ERR_NULLPOINTER;
    o->frames = buffer; o->framesU16 = 1; o->framesTransposed = transposeMode ? 1 : 0; o->framesOnDevice = 0;
    return dh::ERR_SUCCESS;
}
unsigned short* digHoloGetFrameBufferUint16(int h, int* transposeMode) {
    OBJ_OR(h, nullptr);
    if (transposeMode) *transposeMode = o->framesTransposed;
    return o->framesU16 ? (unsigned short*)o->frames : nullptr;
}

// digHolo.h:483-540 / digHolo.cpp:4401-4463, 15073-15121
static int setBatchCommon(Object* o, int batchCount, const void* buf, int u16, int avgCount, int avgMode, int transpose) {
    if (!buf) return dh::ERR_NULLPOINTER;
    o->frames = buf; o->framesU16 = u16; o->framesTransposed = transpose ? 1 : 0; o->framesOnDevice = 0;
    if (batchCount < 1) batchCount = 1;
    if (avgCount < 1) avgCount = 1;
    if (!u16 && (avgMode < 0 || avgMode > 1)) avgMode = 0;
    o->cfg.batchCount = batchCount;
    o->cfg.avgCount = avgCount;
    o->cfg.avgMode = avgMode;
    return dh::ERR_SUCCESS;
}
int digHoloSetBatch(int h, int batchCount, float* buffer) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    return setBatchCommon(o, batchCount, buffer, 0, 1, 0, 0);
}
int digHoloSetBatchAvg(int h, int batchCount, float* buffer, int avgCount, int avgMode) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    return setBatchCommon(o, batchCount, buffer, 0, avgCount, avgMode, 0);
}
int digHoloSetBatchUint16(int h, int batchCount, unsigned short* buffer, int transpose) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    return setBatchCommon(o, batchCount, buffer, 1, 1, 0, transpose);
}
int digHoloSetBatchAvgUint16(int h, int batchCount, unsigned short* buffer, int avgCount, int avgMode, int transpose) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    return setBatchCommon(o, batchCount, buffer, 1, avgCount, avgMode, transpose);
}

// ------------------------------------------------------------ configuration
// digHolo.h:298 / digHolo.cpp:4152 (dimensions must be multiples of 16)
int digHoloConfigSetFrameDimensions(int h, int width, int height) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (width % 16 || height % 16 || width < 0 || height < 0) return dh::ERR_INVALIDDIMENSION;
    o->cfg.frameWidth = width;
    o->cfg.frameHeight = height;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetFrameDimensions(int h, int* width, int* height) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (width) *width = o->cfg.frameWidth;
    if (height) *height = o->cfg.frameHeight;
    return dh::ERR_SUCCESS;
}
// digHolo.h:317 / digHolo.cpp:13856
int digHoloConfigSetFramePixelSize(int h, float pixelSize) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!(pixelSize > 0) || !std::isfinite(pixelSize)) return dh::ERR_INVALIDDIMENSION;
    o->cfg.pixelSize = pixelSize;
    return dh::ERR_SUCCESS;
}
float digHoloConfigGetFramePixelSize(int h) { OBJ_OR(h, 0.f); return o->cfg.pixelSize; }
// digHolo.h:334 / digHolo.cpp:13922
int digHoloConfigSetPolCount(int h, int polCount) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (polCount > 0 && polCount <= dh::POLMAX) { o->cfg.polCount = polCount; return dh::ERR_SUCCESS; }
    return dh::ERR_INVALIDPOLARISATION;
}
int digHoloConfigGetPolCount(int h) { OBJ_OR(h, 0); return o->cfg.polCount; }
// digHolo.h:449
int digHoloConfigSetFillFactorCorrectionEnabled(int h, int enabled) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->cfg.fillFactorCorrection = enabled ? 1 : 0;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetFillFactorCorrectionEnabled(int h) { OBJ_OR(h, 0); return o->cfg.fillFactorCorrection; }
// digHolo.h:551-680 / digHolo.cpp:14826-14910
int digHoloConfigSetBatchCount(int h, int batchCount) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->cfg.batchCount = batchCount < 1 ? 1 : batchCount;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetBatchCount(int h) { OBJ_OR(h, 0); return o->cfg.batchCount; }
int digHoloConfigSetBatchAvgCount(int h, int avgCount) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->cfg.avgCount = avgCount < 1 ? 1 : avgCount;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetBatchAvgCount(int h) { OBJ_OR(h, 0); return o->cfg.avgCount; }
int digHoloConfigSetBatchAvgMode(int h, int avgMode) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->cfg.avgMode = (avgMode < 0 || avgMode >= 3) ? 0 : avgMode;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetBatchAvgMode(int h) { OBJ_OR(h, 0); return o->cfg.avgMode; }
// digHolo.h:599-645 / digHolo.cpp:4468-4520
int digHoloConfigSetBatchCalibration(int h, complex64* cal, int polCount, int batchCount) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (polCount > 0 && batchCount > 0 && cal) {
        o->batchCal.assign((float*)cal, (float*)cal + 2 * (size_t)polCount * batchCount);
        o->batchCalPolCount = polCount;
        o->batchCalCount = batchCount;
        o->batchCalEnabled = 1;
        o->batchCalVersion++;
        return dh::ERR_SUCCESS;
    }
    o->batchCalEnabled = 0;
    o->batchCalVersion++;
    return cal ? dh::ERR_INVALIDARGUMENT : dh::ERR_NULLPOINTER;
}
complex64* digHoloConfigGetBatchCalibration(int h, int* polCount, int* batchCount) {
    OBJ_OR(h, nullptr);
    if (o->batchCal.empty()) { *polCount = 0; *batchCount = 0; return nullptr; }
    *polCount = o->batchCalPolCount;
    *batchCount = o->batchCalCount;
    return (complex64*)o->batchCal.data();
}
int digHoloConfigSetBatchCalibrationEnabled(int h, int enabled) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->batchCalEnabled = enabled ? 1 : 0;
    o->batchCalVersion++;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetBatchCalibrationEnabled(int h) { OBJ_OR(h, 0); return o->batchCalEnabled; }
// digHolo.h:701-749 / digHolo.cpp:14219-14300 (sizes floored to multiples of 16)
int digHoloConfigSetfftWindowSize(int h, int width, int height) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (width < 0 || height < 0) return dh::ERR_INVALIDDIMENSION;
    o->cfg.fftWindowSizeX = 16 * (width / 16);
    o->cfg.fftWindowSizeY = 16 * (height / 16);
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetfftWindowSize(int h, int* width, int* height) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    *width = o->cfg.fftWindowSizeX;
    *height = o->cfg.fftWindowSizeY;
    return dh::ERR_SUCCESS;
}
int digHoloConfigSetfftWindowSizeX(int h, int width) {
    OBJ_OR(h, 0);
    if (width < 0) return 0;
    o->cfg.fftWindowSizeX = 16 * (width / 16);
    return o->cfg.fftWindowSizeX;
}
int digHoloConfigGetfftWindowSizeX(int h) { OBJ_OR(h, 0); return o->cfg.fftWindowSizeX; }
int digHoloConfigSetfftWindowSizeY(int h, int height) {
    OBJ_OR(h, 0);
    if (height < 0) return 0;
    o->cfg.fftWindowSizeY = 16 * (height / 16);
    return o->cfg.fftWindowSizeY;
}
int digHoloConfigGetfftWindowSizeY(int h) { OBJ_OR(h, 0); return o->cfg.fftWindowSizeY; }
// digHolo.h:766 / digHolo.cpp:13520
int digHoloConfigSetFourierWindowRadius(int h, float r) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (r > 0) { o->cfg.apertureSize = r; return dh::ERR_SUCCESS; }
    return dh::ERR_INVALIDDIMENSION;
}
float digHoloConfigGetFourierWindowRadius(int h) { OBJ_OR(h, 0.f); return o->cfg.apertureSize; }
// digHolo.h:786 / digHolo.cpp:14414
int digHoloConfigSetIFFTResolutionMode(int h, int mode) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (mode == 0 || mode == 1) { o->cfg.resolutionIdx = mode; return dh::ERR_SUCCESS; }
    return dh::ERR_INVALIDARGUMENT;
}
int digHoloConfigGetIFFTResolutionMode(int h) { OBJ_OR(h, 0); return o->cfg.resolutionIdx; }
// digHolo.h:814 / digHolo.cpp:14589
int digHoloConfigSetWavelengthCentre(int h, float lambda0) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (lambda0 > 0 && std::isfinite(lambda0)) { o->cfg.wavelengthCentre = lambda0; return dh::ERR_SUCCESS; }
    return dh::ERR_INVALIDARGUMENT;
}
float digHoloConfigGetWavelengthCentre(int h) { OBJ_OR(h, 0.f); return o->cfg.wavelengthCentre; }
// digHolo.h:1205-1255 / digHolo.cpp:13736-14200
int digHoloConfigSetBeamCentre(int h, int axisIdx, int polIdx, float value) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!std::isfinite(value)) return dh::ERR_INVALIDARGUMENT;
    if (polIdx < 0 || polIdx >= o->cfg.polCount) return dh::ERR_INVALIDPOLARISATION;
    if (axisIdx == 0) o->cfg.beamCentreX[polIdx] = value;
    else if (axisIdx == 1) o->cfg.beamCentreY[polIdx] = value;
    else return dh::ERR_INVALIDAXIS;
    return dh::ERR_SUCCESS;
}
float digHoloConfigGetBeamCentre(int h, int axisIdx, int polIdx) {
    OBJ_OR(h, 0.f);
    if (polIdx < 0 || polIdx >= o->cfg.polCount) return 0.f;
    if (axisIdx == 0) return o->cfg.beamCentreX[polIdx];
    if (axisIdx == 1) return o->cfg.beamCentreY[polIdx];
    return 0.f;
}
int digHoloConfigSetTilt(int h, int axisIdx, int polIdx, float value) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!std::isfinite(value)) return dh::ERR_INVALIDARGUMENT;
    if (polIdx < 0 || polIdx >= dh::POLMAX) return dh::ERR_INVALIDPOLARISATION;
    if (axisIdx == 0) o->cfg.zern[polIdx][dh::ZERN_TILTX] = value;
    else if (axisIdx == 1) o->cfg.zern[polIdx][dh::ZERN_TILTY] = value;
    else return dh::ERR_INVALIDAXIS;
    return dh::ERR_SUCCESS;
}
float digHoloConfigGetTilt(int h, int axisIdx, int polIdx) {
    OBJ_OR(h, 0.f);
    if (polIdx < 0 || polIdx >= dh::POLMAX) return 0.f;
    if (axisIdx == 0) return o->cfg.zern[polIdx][dh::ZERN_TILTX];
    if (axisIdx == 1) return o->cfg.zern[polIdx][dh::ZERN_TILTY];
    return 0.f;
}
int digHoloConfigSetDefocus(int h, int polIdx, float value) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (polIdx < 0 || polIdx >= dh::POLMAX) return dh::ERR_INVALIDPOLARISATION;
    o->cfg.zern[polIdx][dh::ZERN_DEFOCUS] = value;
    return dh::ERR_SUCCESS;
}
float digHoloConfigGetDefocus(int h, int polIdx) {
    OBJ_OR(h, 0.f);
    if (polIdx < 0 || polIdx >= dh::POLMAX) return 0.f;
    return o->cfg.zern[polIdx][dh::ZERN_DEFOCUS];
}
// digHolo.h:1270-1326 / digHolo.cpp:13958-14010
int digHoloConfigSetPolLockTilt(int h, int v) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.polLockTilt = v ? 1 : 0; return 0; }
int digHoloConfigGetPolLockTilt(int h) { OBJ_OR(h, 0); return o->cfg.polLockTilt; }
int digHoloConfigSetPolLockDefocus(int h, int v) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.polLockDefocus = v ? 1 : 0; return 0; }
int digHoloConfigGetPolLockDefocus(int h) { OBJ_OR(h, 0); return o->cfg.polLockDefocus; }
int digHoloConfigSetPolLockBasisWaist(int h, int v) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.polLockBasisWaist = v ? 1 : 0; return 0; }
int digHoloConfigGetPolLockBasisWaist(int h) { OBJ_OR(h, 0); return o->cfg.polLockBasisWaist; }
// digHolo.h:1384 / digHolo.cpp:14717 (negative counts are made positive)
int digHoloConfigSetBasisGroupCount(int h, int maxMG) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->cfg.maxMG = maxMG < 0 ? -maxMG : maxMG;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetBasisGroupCount(int h) { OBJ_OR(h, 0); return o->cfg.maxMG; }
// digHolo.h:1404 / digHolo.cpp:14044: the value is written to every polarisation
int digHoloConfigSetBasisWaist(int h, int polIdx, float value) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!(value > 0) || !std::isfinite(value)) return dh::ERR_INVALIDDIMENSION;
    if (polIdx < 0 || polIdx >= dh::POLMAX) return dh::ERR_INVALIDPOLARISATION;
    for (int p = 0; p < o->cfg.polCount; p++) o->cfg.waist[p] = value;
    return dh::ERR_SUCCESS;
}
float digHoloConfigGetBasisWaist(int h, int polIdx) {
    OBJ_OR(h, 0.f);
    if (polIdx < 0 || polIdx >= dh::POLMAX) return 0.f;
    return o->cfg.waist[polIdx];
}
// digHolo.h:1424-1472 / digHolo.cpp:14736-14805, 4750-4765.  The type is
// stored as given and, like the reference, an unknown type or an invalid
// custom matrix processes as Hermite-Gaussian; SetBasisType returns the type.
int digHoloConfigSetBasisTypeHG(int h) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.basisType = 0; return 0; }
int digHoloConfigSetBasisTypeLG(int h) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.basisType = 1; return 0; }
int digHoloConfigSetBasisTypeCustom(int h, int modeCountIn, int modeCountOut, complex64* transform) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!transform) return dh::ERR_NULLPOINTER;
    if (modeCountIn <= 0 || modeCountOut <= 0) return dh::ERR_INVALIDDIMENSION;
    o->cfg.basisType = 2;
    const float* t = reinterpret_cast<const float*>(transform);
    o->basisCustom.assign(t, t + 2 * (size_t)modeCountIn * modeCountOut);
    o->basisCustomIn = modeCountIn;
    o->basisCustomOut = modeCountOut;
    o->basisCustomVersion++;
    return dh::ERR_SUCCESS;
}
int digHoloConfigSetBasisType(int h, int basisType) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->cfg.basisType = basisType;
    return basisType;
}
int digHoloConfigGetBasisType(int h) { OBJ_OR(h, 0); return o->cfg.basisType; }
// digHolo.h:1749-1757: accepted for compatibility; work runs on the GPU
int digHoloConfigSetThreadCount(int h, int threadCount) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (threadCount < 1) threadCount = (int)std::thread::hardware_concurrency();
    o->cfg.threadCount = threadCount;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetThreadCount(int h) { OBJ_OR(h, 0); return o->cfg.threadCount; }
// digHolo.h:1924-1937
int digHoloConfigSetVerbosity(int h, int v) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.verbosity = v; return 0; }
int digHoloConfigGetVerbosity(int h) { OBJ_OR(h, 0); return o->cfg.verbosity; }
// digHolo.h:1808-1818: planning mode 0 (estimate) uses the built-in kernel
// choice; 1-3 (measure, patient, exhaustive) tune the forward and inverse
// kernels by timing on the first batch of each shape (dh_object.cpp)
int digHoloConfigSetFFTWPlanMode(int h, int m) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (m < 0 || m >= 4) return dh::ERR_INVALIDARGUMENT;
    o->cfg.fftwPlanMode = m;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetFFTWPlanMode(int h) { OBJ_OR(h, 0); return o->cfg.fftwPlanMode; }
// digHolo.h:1825 and 1835: the kernel plans play the part of FFTW's wisdom
int digHoloFFTWWisdomForget() { return dh::planForget(); }
int digHoloFFTWWisdomFilename(const char* filename) { return dh::planFilename(filename); }
int digHoloB200GetKernelPlan(int h, int* fwd, int* inv, float* ms) {
    OBJ_OR(h, 0);
    std::lock_guard<std::mutex> guard(o->lock);
    if (!o->preparedValid) return 0;
    return dh::objPlanLookup(*o, fwd, inv, ms);
}
int digHoloB200GetKernelPlanRuns() { return dh::planRuns(); }

// AutoAlign switches (digHolo.h:938-1136)
#define DH_FLAG(NAME, FIELD)                                                                           \
    int digHoloConfigSet##NAME(int h, int v) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.FIELD = v ? 1 : 0; return 0; } \
    int digHoloConfigGet##NAME(int h) { OBJ_OR(h, 0); return o->cfg.FIELD; }
DH_FLAG(AutoAlignBeamCentre, autoAlignCentre)
DH_FLAG(AutoAlignDefocus, autoAlignDefocus)
DH_FLAG(AutoAlignTilt, autoAlignTilt)
DH_FLAG(AutoAlignBasisWaist, autoAlignBasisWaist)
DH_FLAG(AutoAlignFourierWindowRadius, autoAlignFourierWindowRadius)
DH_FLAG(AutoAlignPolIndependence, autoAlignPolIndependence)
DH_FLAG(AutoAlignBasisMulConjTrans, autoAlignBasisMulConjTrans)
#undef DH_FLAG
int digHoloConfigSetAutoAlignTol(int h, float tol) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); o->cfg.autoAlignTol = tol; return 0; }
float digHoloConfigGetAutoAlignTol(int h) { OBJ_OR(h, 0.f); return o->cfg.autoAlignTol; }
int digHoloConfigSetAutoAlignMode(int h, int mode) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (mode < 0 || mode >= 3) return dh::ERR_INVALIDARGUMENT;
    o->cfg.autoAlignMode = mode;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetAutoAlignMode(int h) { OBJ_OR(h, 0); return o->cfg.autoAlignMode; }
int digHoloConfigSetAutoAlignGoalIdx(int h, int goal) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (goal < 0 || goal >= dh::METRIC_COUNT) return dh::ERR_INVALIDARGUMENT;
    o->cfg.autoAlignGoalIdx = goal;
    return dh::ERR_SUCCESS;
}
int digHoloConfigGetAutoAlignGoalIdx(int h) { OBJ_OR(h, 0); return o->cfg.autoAlignGoalIdx; }

// ------------------------------------------------------------ processing
// digHolo.h:1494 / digHolo.cpp:15123 and 4693-4728
complex64* digHoloProcessBatch(int h, int* batchCount, int* modeCount, int* polCount) {
    Object* o = get(h);
    if (!o) { *batchCount = 0; *modeCount = 0; *polCount = 0; return nullptr; }
    const int r = dh::objProcessBatch(*o, 1);
    *batchCount = o->batchCount;
    *polCount = o->polCount;
    *modeCount = dh::objOutputModes(*o);
    if (r != dh::ERR_SUCCESS || o->modeCount <= 0) {
        if (r != dh::ERR_SUCCESS) { *batchCount = 0; *polCount = 0; }
        *modeCount = 0;
        return nullptr;
    }
    return (complex64*)o->hCoefs.ptr;
}
// digHolo.h:1776 / digHolo.cpp (digHoloBenchmark).  Runs digHoloProcessBatch
// on the current batch for about goalDuration seconds (at least three
// batches after one untimed batch) and returns batches per second (host
// clock around the calls, coefficients copied to the host each time, as the
// reference's batch call does).  info (optional, 6 floats,
// DIGHOLO_BENCHMARK_*): FFT, IFFT, APPLYTILT and OVERLAP rates are the
// batches per second of this build's forward and inverse kernels (device
// time; the IFFT, tilt removal and overlap are one stage here), BASIS the
// rate of a full HG basis computation, TOTAL the frames per second.
float digHoloBenchmark(int h, float goalDuration, float* info) {
    OBJ_OR(h, 0.f);
    if (dh::objProcessBatch(*o, 1) != dh::ERR_SUCCESS) return 0.f;
    const int saveTiming = o->timing;
    o->timing = 1;
    float st[3];
    dh::objStageTimes(*o, st);
    int calls = 0;
    const auto t0 = std::chrono::steady_clock::now();
    double el = 0.0;
    do {
        if (dh::objProcessBatch(*o, 1) != dh::ERR_SUCCESS) { o->timing = saveTiming; return 0.f; }
        calls++;
        el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } while (calls < 3 || el < goalDuration);
    dh::objStageTimes(*o, st);
    o->timing = saveTiming;
    const float rate = (float)(calls / el);
    if (info) {
        const float n = st[2] > 0 ? st[2] : 1.f;
        const float fwd = st[0] > 0 ? 1e3f * n / st[0] : 0.f;
        const float inv = st[1] > 0 ? 1e3f * n / st[1] : fwd;
        info[0] = fwd;
        info[1] = inv;
        info[2] = inv;
        info[4] = inv;
        info[5] = rate * (float)o->batchCount;
        // the basis: one recomputation for the current waists, timed on the host
        const auto b0 = std::chrono::steady_clock::now();
        o->basisNx = -1;   // force the recomputation
        const int rb = dh::objUpdateBasis(*o);
        const double bt = std::chrono::duration<double>(std::chrono::steady_clock::now() - b0).count();
        info[3] = (rb == dh::ERR_SUCCESS && bt > 0) ? (float)(1.0 / bt) : 0.f;
    }
    return rate;
}

// digHolo.h:1670-1706 / digHolo.cpp:15146-15200
int digHoloProcessFFT(int h) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); return dh::objFFT(*o); }
int digHoloProcessIFFT(int h) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); return dh::objIFFT(*o); }
int digHoloProcessRemoveTilt(int h) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); return dh::objApplyTilt(*o); }
int digHoloProcessBasisExtractCoefs(int h) { OBJ_OR(h, dh::ERR_INVALIDHANDLE); return dh::objOverlap(*o); }

// digHolo.h:1603 / digHolo.cpp:15252 and 4827
complex64* digHoloBasisGetCoefs(int h, int* batchCount, int* modeCount, int* polCount) {
    Object* o = get(h);
    if (!o || !o->processedOverlap || o->modeCount <= 0 || !o->hCoefs.ptr) {
        *batchCount = 0; *modeCount = 0; *polCount = 0;
        return nullptr;
    }
    *batchCount = o->batchCount;
    *modeCount = dh::objOutputModes(*o);
    *polCount = o->polCount;
    return (complex64*)o->hCoefs.ptr;
}

// digHolo.h:1549 / digHolo.cpp:15343 and 4930-4981
complex64* digHoloGetFields(int h, int* batchCount, int* polCount, float** x, float** y, int* width, int* height) {
    Object* o = get(h);
    if (!o || !o->processedTilt || dh::objFieldsToHost(*o, 1) != dh::ERR_SUCCESS) {
        *batchCount = 0; *polCount = 0; *x = nullptr; *y = nullptr; *width = 0; *height = 0;
        return nullptr;
    }
    o->hX = o->geo.x;
    o->hY = o->geo.y;
    *batchCount = o->batchCount;
    *polCount = o->polCount;
    *x = o->hX.data();
    *y = o->hY.data();
    *width = o->geo.nx;
    *height = o->geo.ny;
    return (complex64*)o->hFields.ptr;
}

// digHolo.h:1568 / digHolo.cpp:4880-4928
int digHoloGetFields16(int h, int* batchCount, int* polCount, short** fieldR, short** fieldI, float** fieldScale,
                       float** x, float** y, int* width, int* height) {
    Object* o = get(h);
    if (!o) return dh::ERR_INVALIDHANDLE;
    if (!o->processedTilt || dh::objFieldsToHost(*o, 0) != dh::ERR_SUCCESS) {
        *batchCount = 0; *polCount = 0; *fieldR = nullptr; *fieldI = nullptr; *fieldScale = nullptr;
        *x = nullptr; *y = nullptr; *width = 0; *height = 0;
        return dh::ERR_NULLPOINTER;
    }
    const size_t n = (size_t)o->batchCount * o->polCount * o->geo.nx * o->geo.ny;
    o->hX = o->geo.x;
    o->hY = o->geo.y;
    *batchCount = o->batchCount;
    *polCount = o->polCount;
    *fieldR = o->hFieldR.as<short>();
    *fieldI = o->hFieldR.as<short>() + n;
    // DIGHOLO_ANALYSIS[IFFT][MAXABS][pol][batch]
    *fieldScale = o->hStats.as<float>() + 3 * o->polCount * (o->batchCount * o->avgCount + 1);
    *x = o->hX.data();
    *y = o->hY.data();
    *width = o->geo.nx;
    *height = o->geo.ny;
    return dh::ERR_SUCCESS;
}

// digHolo.h:1659 / digHolo.cpp:4767-4805.  Plane 1 (reconstructed field)
// comes from the batch path; plane 0 (the Fourier plane of the camera) is
// computed from the batch's frames on the first request (the full R2C plane
// and its analysis, digHolo.cpp:6931-6980).  The batch-sum intensities have
// W H floats per polarisation (FFT window size), as in the reference.
int digHoloBatchGetSummary(int h, int planeIdx, int* parameterCount, int* totalCount, int* polCount, float** parameters,
                           int* pixelCountX, int* pixelCountY, float** xAxis, float** yAxis, float** totalIntensity) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (planeIdx < 0 || planeIdx > 1) return dh::ERR_INVALIDDIMENSION;
    if (!o->processedTilt) return dh::ERR_NULLPOINTER;
    if (planeIdx == 0) {
        if (dh::objFourierToHost(*o, 0) != dh::ERR_SUCCESS) return dh::ERR_ERROR;
        *parameterCount = dh::ANALYSIS_COUNT;
        *totalCount = o->lastFwd.frameCount + 1;
        *polCount = o->polCount;
        *parameters = o->hFftStats.as<float>();
        *pixelCountX = o->geo.W / 2 + 1;
        *pixelCountY = o->geo.H;
        *xAxis = o->hKx.data();
        *yAxis = o->hKy.data();
        *totalIntensity = o->hFftBatchSum.as<float>();
        return dh::ERR_SUCCESS;
    }
    if (dh::objStatsToHost(*o) != dh::ERR_SUCCESS) return dh::ERR_ERROR;
    o->hX = o->geo.x;
    o->hY = o->geo.y;
    *parameterCount = dh::ANALYSIS_COUNT;
    *totalCount = o->batchCount * o->avgCount + 1;
    *polCount = o->polCount;
    *parameters = o->hStats.as<float>();
    *pixelCountX = o->geo.nx;
    *pixelCountY = o->geo.ny;
    *xAxis = o->hX.data();
    *yAxis = o->hY.data();
    *totalIntensity = o->hBatchSum.as<float>();
    return dh::ERR_SUCCESS;
}

// digHolo.h:1718 / digHolo.cpp:4362-4380, 15554-15564.  The R2C planes
// [batch][pol][H][W/2+1] of the last batch, computed from its frames on the
// first request; as the reference does, *width reports the FFT window width
// W (the rows hold W/2+1 values).  Null and zero sizes before any batch.
complex64* digHoloGetFourierPlaneFull(int h, int* batchCount, int* polCount, int* width, int* height) {
    Object* o = get(h);
    if (!o) return nullptr;
    if (!o->processedTilt || dh::objFourierToHost(*o, 1) != dh::ERR_SUCCESS) {
        *batchCount = *polCount = *width = *height = 0;
        return nullptr;
    }
    *batchCount = o->lastFwd.frameCount;
    *polCount = o->polCount;
    *width = o->geo.W;
    *height = o->geo.H;
    return (complex64*)o->hFourier.ptr;
}

// digHolo.h:1732 / digHolo.cpp:4370-4390.  The window is returned in the
// low-resolution layout [batch][pol][h][w] in both resolution modes.
complex64* digHoloGetFourierPlaneWindow(int h, int* batchCount, int* polCount, int* width, int* height) {
    Object* o = get(h);
    if (!o || !o->processedIFFT || dh::objWindowToHost(*o) != dh::ERR_SUCCESS) {
        *batchCount = 0; *polCount = 0; *width = 0; *height = 0;
        return nullptr;
    }
    *batchCount = o->batchCount;
    *polCount = o->polCount;
    *width = o->geo.w;
    *height = o->geo.h;
    return (complex64*)o->hWindow.ptr;
}

// ------------------------------------------------------------ metrics and AutoAlign
// digHolo.h:1152 / digHolo.cpp:14989 and 13012-13016
float digHoloAutoAlign(int h) {
    OBJ_OR(h, 0.0f);
    return dh::objAutoAlign(*o);
}
// digHolo.h:1163 / digHolo.cpp:15014: the metric averaged over wavelengths
float digHoloAutoAlignGetMetric(int h, int metricIdx) {
    OBJ_OR(h, 0.0f);
    if (metricIdx < 0 || metricIdx >= dh::METRIC_COUNT) return 0.0f;
    return o->autoAlignMetrics[metricIdx][1];
}
// digHolo.h:1174 / digHolo.cpp:15001: [wavelength 0, average]
float* digHoloAutoAlignGetMetrics(int h, int metricIdx) {
    OBJ_OR(h, nullptr);
    if (metricIdx < 0 || metricIdx >= dh::METRIC_COUNT) return nullptr;
    return o->autoAlignMetrics[metricIdx];
}
// digHolo.h:1185 / digHolo.cpp:15043 and 12214-12230
int digHoloAutoAlignCalcMetrics(int h) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    std::lock_guard<std::mutex> g(o->lock);
    return dh::objCalcMetrics(*o);
}

// ------------------------------------------------------------ extensions
// No counterpart in the reference: device-resident use without host copies.

// Runs the batch path on frames already in device memory (digHoloSetBatch*
// given a device pointer) and leaves every output on the device; returns
// without waiting for the GPU.
int digHoloB200ProcessBatchDevice(int h) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    return dh::objProcessBatch(*o, 0);
}
// Device pointer to the coefficients [batch][pol*mode] of the last batch.
complex64* digHoloB200GetCoefsDevice(int h, int* batchCount, int* modeCount, int* polCount) {
    Object* o = get(h);
    if (!o || o->modeCount <= 0 || !o->dCoefs.ptr) { *batchCount = 0; *modeCount = 0; *polCount = 0; return nullptr; }
    *batchCount = o->batchCount;
    *modeCount = dh::objOutputModes(*o);
    *polCount = o->polCount;
    return reinterpret_cast<complex64*>(const_cast<float2*>(dh::objOutputCoefs(*o)));
}
// Waits for the handle's GPU work; returns a CUDA error as DIGHOLO_ERROR_ERROR.
int digHoloB200Synchronize(int h) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!o->stream) return dh::ERR_SUCCESS;
    if (cudaStreamSynchronize(o->stream) != cudaSuccess) return dh::ERR_ERROR;
    return dh::objCheckStatus(*o);
}
// Keep the float field -conj(A.ref) before int16 rounding (off by default).
int digHoloB200SetKeepField32(int h, int enable) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->keepField32 = enable ? 1 : 0;
    return dh::ERR_SUCCESS;
}
// Copies the float fields of the last batch to host memory ([batch][pol][h][w]).
complex64* digHoloB200GetFields32(int h, int* batchCount, int* polCount, int* width, int* height) {
    Object* o = get(h);
    if (!o || !o->keepField32 || !o->processedTilt || !o->dField32.ptr) {
        *batchCount = 0; *polCount = 0; *width = 0; *height = 0;
        return nullptr;
    }
    const size_t n = (size_t)o->batchCount * o->polCount * o->geo.nx * o->geo.ny;
    if (!o->hFields.ensure(n * sizeof(float2))) return nullptr;
    if (cudaMemcpy(o->hFields.ptr, o->dField32.ptr, n * sizeof(float2), cudaMemcpyDeviceToHost) != cudaSuccess) return nullptr;
    *batchCount = o->batchCount;
    *polCount = o->polCount;
    *width = o->geo.nx;
    *height = o->geo.ny;
    return (complex64*)o->hFields.ptr;
}
// Runs the handle's GPU work on `stream` (a cudaStream_t owned by the caller;
// nullptr restores a private stream).  Call before the first processing.
int digHoloB200SetStream(int h, void* stream) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (o->stream && !o->userStream) {
        cudaStreamSynchronize(o->stream);
        cudaStreamDestroy(o->stream);
    }
    o->stream = (cudaStream_t)stream;
    o->userStream = stream ? 1 : 0;
    return dh::ERR_SUCCESS;
}
// Enables CUDA-event timing of the forward and inverse kernels of a batch
// processed as one launch each (device-resident frames).
int digHoloB200SetTiming(int h, int enable) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->timing = enable ? 1 : 0;
    return dh::ERR_SUCCESS;
}
// CUDA-graph replay of device-frame batches (on by default): 0 launches
// every batch directly and releases the captured graphs.
int digHoloB200SetGraphs(int h, int enable) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    std::lock_guard<std::mutex> guard(o->lock);
    o->useGraphs = enable ? 1 : 0;
    o->graphFailures = 0;
    if (!enable) {
        if (o->stream) cudaStreamSynchronize(o->stream);
        dh::objReleaseGraphs(*o);
    }
    return dh::ERR_SUCCESS;
}
int digHoloB200GetGraphCount(int h) {
    OBJ_OR(h, 0);
    return (int)o->graphs.size();
}
// Kernel times of the batches processed with timing on since the last call:
// out[0] forward-kernel ms (sum), out[1] inverse-kernel ms (sum), out[2] count.
int digHoloB200GetStageTimes(int h, float* out3) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    return dh::objStageTimes(*o, out3);
}
// Window geometry of the last processed batch: out[0..5] = W, H (FFT window),
// w, h (IFFT window), nx, ny (reconstructed field); out[6..7] = FFT window
// corner x, y of polarisation 0; out[8..9] = SX, SY of polarisation 0.
int digHoloB200GetGeometry(int h, int* out10) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    const dh::Geometry& g = o->geo;
    const int v[10] = {g.W, g.H, g.w, g.h, g.nx, g.ny, g.cx[0], g.cy[0], g.SX[0], g.SY[0]};
    for (int i = 0; i < 10; i++) out10[i] = v[i];
    return dh::ERR_SUCCESS;
}
// Selects the forward kernel: 0 = fastest available (default), 1 = always
// the shared-memory kernel (used by the tests to cover both).
int digHoloB200SetForwardKernel(int h, int kernel) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (kernel < 0 || kernel > 5) return dh::ERR_INVALIDARGUMENT;
    o->forwardKernel = kernel;
    return dh::ERR_SUCCESS;
}
int digHoloB200SetInverseKernel(int h, int kernel) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (kernel < 0 || kernel > 3) return dh::ERR_INVALIDARGUMENT;
    o->inverseKernel = kernel;
    return dh::ERR_SUCCESS;
}
// Inverse kernel used by the last batch: 1 block per unit, 2 warp per unit,
// 3 full-resolution field kernel + overlap kernel, 4 full-resolution bands,
// 5 fused into the tensor-core forward kernel.
int digHoloB200GetInverseKernel(int h) {
    OBJ_OR(h, 0);
    return o->lastInverseKernel;
}
int digHoloB200SetOverlapKernel(int h, int kernel) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (kernel < 0 || kernel > 1) return dh::ERR_INVALIDARGUMENT;
    o->overlapKernel = kernel;
    return dh::ERR_SUCCESS;
}
// Overlap used by the last batch: 1 FP32 CUDA cores, 2 split-BF16 tensor cores.
int digHoloB200GetOverlapKernel(int h) {
    OBJ_OR(h, 0);
    return o->lastOverlapKernel;
}
// Forward kernel used by the last batch: 1 generic, 2 register, 3 TMA-fed,
// 4 tensor-core row DFT (uint16 frames), 5 full planes.
int digHoloB200GetForwardKernel(int h) {
    OBJ_OR(h, 0);
    return o->lastForwardKernel;
}
// Gradient of IL = 10 log10(sum |c|^2) + const with respect to
// [pol][tiltX, tiltY, defocus, beamCentreX, beamCentreY, waist] at the current
// configuration (Fourier-window selection held fixed), from one batch pass
// and its adjoint on the GPU; il = 10 log10(sum |c|^2).
int digHoloB200AutoAlignGradient(int h, float* grad12, float* il) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!grad12) return dh::ERR_NULLPOINTER;
    return dh::objAlignGradient(*o, grad12, il);
}
// Gradient of a metric (0 IL, 1 MDL, both in dB) with the layout of
// digHoloB200AutoAlignGradient; *value = the metric at the current settings.
int digHoloB200AutoAlignGradientMetric(int h, int metricIdx, float* grad12, float* value) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    if (!grad12) return dh::ERR_NULLPOINTER;
    if (metricIdx != 0 && metricIdx != 1) return dh::ERR_INVALIDARGUMENT;
    return dh::objAlignGradientMetric(*o, metricIdx, grad12, value);
}
// Holds the FFT window and the Fourier-window selection and mask at the
// current settings (enable = 1) while the beam-centre phase, the reference
// wave and the basis keep following the configuration; 0 releases them.
int digHoloB200FreezeWindow(int h, int enable) {
    OBJ_OR(h, dh::ERR_INVALIDHANDLE);
    o->useSnaps = enable ? 1 : 0;
    if (enable) o->fftSnap = o->ifftSnap = o->cfg;
    o->preparedValid = 0;
    return dh::ERR_SUCCESS;
}
// Gradient-driven AutoAlign (goal IL): quasi-Newton on the adjoint gradient.
// Returns the goal metric of the final configuration; the metrics are read
// with digHoloAutoAlignGetMetric(s) as after digHoloAutoAlign.
float digHoloB200AutoAlignAdjoint(int h) {
    OBJ_OR(h, 0.0f);
    return dh::objAutoAlignAdjoint(*o);
}
// Number of batch evaluations the last digHoloAutoAlign ran.
int digHoloB200GetAutoAlignEvaluations(int h) {
    OBJ_OR(h, 0);
    return o->alignEvaluations;
}
// Last error message of the handle (empty when none).
const char* digHoloB200GetLastError(int h) {
    OBJ_OR(h, "invalid handle");
    return o->lastError.c_str();
}

}  // extern "C"
