// Per-handle state of the digholo_b200 runtime: the user configuration (the
// fields of digHoloConfig, digHolo.cpp:3323-3372), the derived window
// geometry, the device buffers and the host mirrors returned to callers.
#pragma once
#include <cstdio>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>
#include <memory>
#include <vector>

#include "dh_params.h"

struct DhEigen;

namespace dh {

// Error codes and constants of the public interface (digHolo.h:171-182, 1363-1372, 1624-1631).
enum {
    ERR_SUCCESS = 0, ERR_ERROR = 1, ERR_INVALIDHANDLE = 2, ERR_NULLPOINTER = 3,
    ERR_INVALIDDIMENSION = 5, ERR_INVALIDPOLARISATION = 6, ERR_INVALIDAXIS = 7,
    ERR_INVALIDARGUMENT = 8, ERR_MEMORYALLOCATION = 9
};
constexpr int POLMAX = 2;
constexpr int ANALYSIS_COUNT = 7;
constexpr int METRIC_COUNT = 9;
constexpr int METRIC_IL = 0, METRIC_MDL = 1, METRIC_DIAG = 2, METRIC_SNRAVG = 3, METRIC_DIAGBEST = 4,
              METRIC_DIAGWORST = 5, METRIC_SNRBEST = 6, METRIC_SNRWORST = 7, METRIC_SNRMG = 8;
constexpr int ZERN_TILTX = 1, ZERN_TILTY = 2, ZERN_DEFOCUS = 4;

struct Config {
    int frameWidth = 320;
    int frameHeight = 256;
    float pixelSize = 20e-6f;
    float apertureSize = 0.4f;          // Fourier window radius, degrees
    int resolutionIdx = 0;              // 0 full resolution, 1 window-size IFFT
    float waist[POLMAX] = {510.f, 510.f};
    float zern[POLMAX][6] = {{0, -0.75f, 0.75f, 0, 0, 0}, {0, -0.75f, 0.75f, 0, 0, 0}};
    float beamCentreX[POLMAX] = {0.f, 0.f};
    float beamCentreY[POLMAX] = {0.f, 0.f};
    int batchCount = 0;
    int avgCount = 1;
    int avgMode = 0;
    float wavelengthCentre = 1565e-9f;
    // first and last wavelength of a multi-wavelength batch (0: the centre
    // wavelength alone): the IFFT window spans the Fourier windows of both
    float lambdaRange[2] = {0.f, 0.f};
    int wavelengthOrdering[2] = {0, 0};
    int polLockTilt = 0;
    int polLockBasisWaist = 1;
    int polLockDefocus = 0;
    int polCount = 1;
    int autoAlignTilt = 1, autoAlignDefocus = 1, autoAlignCentre = 1, autoAlignBasisWaist = 1;
    int autoAlignFourierWindowRadius = 1, autoAlignPolIndependence = 0, autoAlignBasisMulConjTrans = 0;
    float autoAlignTol = 0.f;
    int autoAlignMode = 0;
    int fillFactorCorrection = 1;
    int autoAlignGoalIdx = 0;
    int fftWindowSizeX = 0;
    int fftWindowSizeY = 0;
    int fftwPlanMode = 0;
    int maxMG = 0;
    int basisType = 0;
    int verbosity = 0;
    int threadCount = 1;
};

// Grow-only device allocation.  Every (re)allocation or release advances
// devBufGeneration(), which invalidates the captured batch graphs.
unsigned long long devBufGeneration();
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n);
    void release();
    ~DevBuf() { release(); }
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// Grow-only pinned host allocation (host mirrors of returned arrays).
struct HostBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool ensure(size_t n);
    void release();
    ~HostBuf() { release(); }
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// Geometry of the FFT and IFFT windows, computed with the reference's
// float32 arithmetic (digHolo.cpp:7267-7378, 7868-8048, 8183-8203).
struct Geometry {
    int W = 0, H = 0;                 // FFT window
    int cx[POLMAX] = {0, 0}, cy[POLMAX] = {0, 0};
    int w = 0, h = 0;                 // IFFT window
    int SX[POLMAX] = {0, 0}, SY[POLMAX] = {0, 0};
    int nx = 0, ny = 0;               // reconstructed field
    std::vector<float> kx, ky;        // fftshifted Fourier axes (W, H)
    std::vector<float> x, y;          // reconstructed-plane axes (nx, ny)
    std::vector<float> xFull, yFull;  // FFT-window camera axes (W, H)
};

struct Object {
    Config cfg;
    std::mutex lock;

    // frame source (digHoloSetBatch* store the pointer, digHolo.cpp:4401-4463)
    const void* frames = nullptr;
    int framesU16 = 0;
    int framesTransposed = 0;
    int framesOnDevice = 0;

    // batch calibration (digHolo.cpp:4468-4500)
    std::vector<float> batchCal;  // [pol][count] complex interleaved
    int batchCalPolCount = 0, batchCalCount = 0, batchCalEnabled = 0;

    // processed state
    int batchCount = 0, avgCount = 1, polCount = 1;
    int modeCount = 0;
    int processedFFT = 0, processedIFFT = 0, processedTilt = 0, processedOverlap = 0;
    Geometry geo;

    // device state
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evCopy[2] = {nullptr, nullptr};
    // the second polarisation's window copies run on their own stream (a
    // second DMA queue next to the first)
    cudaStream_t copyStream2 = nullptr;
    cudaEvent_t evCopy2[2] = {nullptr, nullptr};
    // coefficients of finished chunks leave for the host on their own stream
    // (the device-to-host DMA direction) while later chunks' frames arrive
    cudaStream_t d2hStream = nullptr;
    cudaEvent_t evChunk[2] = {nullptr, nullptr};
    cudaEvent_t evD2H = nullptr;
    cudaEvent_t evStart = nullptr, evStop = nullptr;
    int userStream = 0;                 // stream supplied by digHoloB200SetStream (not owned)
    int timing = 0;                     // record per-stage events in ProcessBatch
    // device-frame batches replayed as CUDA graphs (digHoloB200SetGraphs):
    // key = every launch argument, exec = the captured forward + inverse launches
    struct BatchGraph {
        std::vector<unsigned char> key;
        cudaGraphExec_t exec = nullptr;
        int fwdKernel = 0, invKernel = 0, ovlKernel = 0;
    };
    std::vector<BatchGraph> graphs;
    std::vector<std::vector<unsigned char>> graphPending;   // settled argument sets (frame pointer zeroed)
    int useGraphs = 1, graphFailures = 0;
    std::vector<cudaEvent_t> evStage;   // 3 events per timed batch since the last read
    int evStageUsed = 0;
    // inputs of the last prepare(): geometry and uploads are reused while they match
    Config preparedCfg;
    int preparedValid = 0, preparedKeep32 = -1, preparedU16 = -1, batchCalVersion = 0, preparedBatchCal = -1;
    DevBuf dTwiddle, dFrames, dWindow, dFieldR, dFieldI, dField32, dStats, dCoefs;
    DevBuf dWindowAvg;                  // frame averaging: the windows of all batch x avg frames
    // output basis (digHoloConfigSetBasisType*): the custom matrix as given
    // ([in][out] complex), the device matrix of the active transform
    // ([dimIn][dimOut]) with the settings it was built for, and the
    // coefficients in that basis [batch][pol][modeCountOut]
    std::vector<float> basisCustom;
    int basisCustomIn = 0, basisCustomOut = 0, basisCustomVersion = 0;
    DevBuf dBasisT, dCoefsOut;
    int basisTType = -1, basisTModes = -1, basisTVersion = -1, basisDimIn = 0;
    int basisActive = 0;                // 0 HG (the overlap's coefficients), 1 LG, 2 custom
    int modeCountOut = 0;
    DevBuf dKx, dKy, dX, dY, dRef, dRefF, dTables, dHgX, dHgY, dHgScaleX, dHgScaleY, dBasisAxis, dBatchCal, dFieldsC64;
    // basis cache key
    int basisNx = 0, basisNy = 0, basisMG = 0;
    float basisWaist[POLMAX] = {0.f, 0.f};
    float basisPsx = 0.f, basisPsy = 0.f;
    int basisPolCount = 0;
    int keepField32 = 0;
    // power meter / AutoAlign
    DevBuf dMetricA, dMetricG, dCoefsBackup, dAlignFrames;
    DevBuf dDigits;                     // tensor-core row DFT digits (uint16 frames)
    // Fourier planes of the last batch (on request): the frame source the
    // batch was processed from, the planes, their statistics and batch sum
    DhFwdParams lastFwd;
    int lastFwdValid = 0, fourierValid = 0;
    float lastFourierR2 = 0.f;
    DevBuf dFourier, dFftStats, dFftBatchSum;
    HostBuf hFourier, hFftStats, hFftBatchSum;
    std::vector<float> hKx, hKy;
    int digitsValid = 0;
    DevBuf dBigScratch;                 // band kernels: partial statistics and coefficients, prepared Hx
    DevBuf dSnap[16];                   // AutoAlign parameter estimate: planes, sums, fields, tables
    DevBuf dTransRaw, dTransFrames;     // transposed uint16 input: raw host copy, converted frames
    // adjoint AutoAlign scratch: derivative windows and fields, float bases, partial sums
    DevBuf dGradW, dGradV, dGradScratch, dGradBasis, dGradOut, dGradTab, dGradWeights;
    double alignMdlDb = 0.0;   // MDL of the batch state the MDL gradient weights belong to
    HostBuf hGradOut;
    DhEigen* eigen = nullptr;
    int alignEvaluations = 0;
    // stage snapshots used while AutoAlign runs: the FFT window comes from
    // fftSnap and the Fourier-window selection from ifftSnap
    int useSnaps = 0;
    Config fftSnap, ifftSnap;
    // forward kernel choice: 0 automatic (TMA-fed, then register, then
    // generic), 1 generic, 2 register, 3 TMA-fed only; and the one that ran last
    int forwardKernel = 0;
    int lastForwardKernel = 0;
    // inverse kernel choice: 0 automatic (warp-per-unit kernel for 16/32-pixel
    // low-resolution fields, else the block kernel), 1 block kernel
    int inverseKernel = 0;
    int lastInverseKernel = 0;
    // overlap of full-resolution fields: 0 tensor cores (split-BF16) where the
    // shape allows, 1 FP32 CUDA cores; and the one that ran last (1 FP32, 2 tensor)
    int overlapKernel = 0;
    int lastOverlapKernel = 0;
    int quietErrors = 0;                // kernel planner trials: launch failures are expected, not printed
    int* hStatus = nullptr;             // host-mapped failure flag written by the kernels
    int* dStatus = nullptr;             // its device address

    // host mirrors
    HostBuf hCoefs, hFields, hFieldR, hFieldI, hStats, hStatsFFT, hWindow, hBatchSum;
    HostBuf hUpload;                    // pinned staging of the per-configuration tables
    cudaEvent_t evUpload = nullptr;     // the last staged upload has left
    std::vector<float> hX, hY;
    // wavelengths (digHoloConfigSetWavelengths*, digHolo.cpp:6578-6690):
    // the pending array and the one in use after the next update
    std::vector<float> wavelengthsNew, wavelengths;
    int wavelengthsValid = 0;
    DevBuf dSweepFrames, dAccCoefs, dAccCoefsOut, dAccFieldR, dAccFieldI, dAccField32, dAccStats;
    // reference-wave calibration (digHoloConfigSetRefCalibration*,
    // digHolo.cpp:5309-5540): the stored per-pixel factors [L][height][width]
    std::vector<float> refCal;
    int refCalWidth = 0, refCalHeight = 0, refCalCount = 0, refCalEnabled = 0;
    int refCalGen = 0;                  // advanced by every calibration setter
    DevBuf dRefCalFrames;               // the stored factors on the device
    int refCalFramesGen = -1;
    DevBuf dRefCalScratch, dRefCalTables;
    // reconstructed calibration planes [pol][ny][nx], one per calibration
    // item, wavelength and geometry in use (key: every input of the planes)
    struct RefCalPlanes {
        std::vector<unsigned char> key;
        DevBuf planes;
    };
    std::vector<std::unique_ptr<RefCalPlanes>> refCalPlanes;
    HostBuf hRefCalFields;
    std::vector<float> hRefCalX, hRefCalY;
    // during a multi-wavelength batch: the sub-batch's wavelength index and
    // the batch calibration as the caller set it (the sub-batches rewrite it)
    int sweepLambda = -1;
    float sweepCentre = 0.f;
    const std::vector<float>* batchCalCaller = nullptr;
    int batchCalCallerCount = 0, batchCalCallerPol = 0;
    // frames loaded by digHoloSetFrameBufferFromFile (owned, float32)
    std::vector<float> ownFrames;
    // digHoloConfigBackupSave / Load
    Config cfgBackup;
    int cfgBackupValid = 0;
    float* zernRows[POLMAX] = {nullptr, nullptr};   // digHoloConfigGetZernCoefs
    HostBuf hBasisFields;                           // digHoloBasisGetFields
    float autoAlignMetrics[METRIC_COUNT][2] = {};
    int metricsValid = 0;
    std::string lastError;
};

// Error reporting shared by the runtime files: the message is kept for
// digHoloB200GetLastError and printed at verbosity >= 1 (CUDA errors always).
inline int fail(Object& o, int code, const char* what) {
    o.lastError = what;
    if (o.cfg.verbosity >= 1) { fprintf(stderr, "digholo_b200: %s\n", what); fflush(stderr); }
    return code;
}
inline int failCuda(Object& o, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    o.lastError = m;
    if (!o.quietErrors) {
        fprintf(stderr, "digholo_b200: %s\n", m.c_str());
        fflush(stderr);
    }
    return ERR_ERROR;
}
#define DH_CUDA(o, call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return failCuda(o, e_, #call); } while (0)

// Runtime entry points used by the C ABI layer.
int objInitDevice(Object& o);
int objFFT(Object& o);
int objIFFT(Object& o);
int objApplyTilt(Object& o);
int objOverlap(Object& o);
int objProcessBatch(Object& o, int syncCoefs);
int objCoefsToHost(Object& o);
int objFieldsToHost(Object& o, int complexOut);
int objStatsToHost(Object& o);
int objFourierToHost(Object& o, int withPlane);
int objWindowToHost(Object& o);
int objStageTimes(Object& o, float* ms);
int objUpdateBasis(Object& o);
int objProcessForAlign(Object& o);
int objCheckStatus(Object& o);
void objReleaseGraphs(Object& o);
// Kernel planner (plan modes above ESTIMATE): process-wide table of tuned
// kernel choices, saved to and loaded from the wisdom file.
int planForget();
int planFilename(const char* filename);
int planRuns();
int objPlanLookup(Object& o, int* forwardKernel, int* inverseKernel, float* ms);
// The coefficients the API returns: in the configured basis after a batch
// (modeCountOut modes per polarisation), else the HG coefficients.
const float2* objOutputCoefs(const Object& o);
int objOutputModes(const Object& o);
int objInverseAux(Object& o, const float2* window, int frameCount, float2* field32, short* scratchR, short* scratchI,
                  float* scratchStats);
int objBasisFloat(Object& o, int modes, float* outX, float* outY, short* scratch16, float* scratchScale);
int objAlignGradient(Object& o, float* grad12, float* ilOut);
int objAlignGradientMetric(Object& o, int metric, float* grad12, float* valueOut);
enum { ALIGN_EVAL_FULL = 0, ALIGN_EVAL_VALUE = 1, ALIGN_EVAL_GRADIENT = 2 };
int objAlignEvaluate(Object& o, int metric, int stage, float* grad12, float* valueOut);
int objMdlWeights(Object& o, float2* W, double* mdlDb);
float objAutoAlignAdjoint(Object& o);
int objCalcMetrics(Object& o);
float objAutoAlign(Object& o);
// The wavelength array in use (digHoloWavelengthUpdate, digHolo.cpp:7823-7862).
void objWavelengthUpdate(Object& o);
// Reference-wave calibration (dh_refcal.cpp).
bool objRefCalApplies(const Object& o);
int objRefCalCheckShape(Object& o, const DhInvParams& ip);
int objRefCalPlanes(Object& o, int item, const float2** out, bool lookupOnly);
int objRefCalFieldsToHost(Object& o);

// Geometry helpers (host, float32 emulation of the reference).
void fftWindowGeometry(const Config& c, int polCount, Geometry& g);
void ifftWindowGeometry(const Config& c, int polCount, Geometry& g);
void referenceWave(const Config& c, int polCount, const Geometry& g, std::vector<short>& out,
                   std::vector<float>* outF = nullptr);
void windowFactors(const Config& c, const Config& live, const Geometry& g, int polCount, std::vector<float>& adj);
bool isPow2(int v);
int ilog2(int v);

}  // namespace dh
