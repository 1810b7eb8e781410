/*
 * digHolo.h -- C ABI of digholo_b200 (libdigholo_b200.so).
 *
 * digholo_b200 runs the digHolo batch path -- camera frames -> FFT of the
 * window around each beam -> off-axis Fourier window -> IFFT -> reference
 * tilt/defocus removal -> Hermite-Gaussian modal overlap -- as sm_100a CUDA
 * kernels on one B200.  The entry points below keep the names, argument
 * meaning, clamping and error returns of the digHolo C interface; each one
 * cites the declaration it replaces in the reference's digHolo.h.  Unlike
 * the reference's Linux build (where EXT_C is empty and the exports are
 * C++-mangled), every name here is exported with C linkage.
 *
 * Ownership follows the reference: frame buffers passed to digHoloSetBatch*
 * stay owned by the caller and are read during processing (host or device
 * pointers both work); returned arrays are host buffers owned by the handle
 * and valid until the next processing or configuration call on it.
 *
 * The digHoloB200* functions at the end have no counterpart in the
 * reference: they serve callers whose frames are already in device memory.
 *
 * The library also exports every reference entry point under its
 * C++-mangled name (e.g. _Z13digHoloCreatev for digHoloCreate), as the
 * reference's Linux build names them (digHolo.h:148-156), so programs
 * compiled with g++ against the reference's header link and run unchanged.
 * Defining DIGHOLO_CXX_LINKAGE before including this header in C++ declares
 * the functions with C++ linkage, i.e. under those names.
 */
#ifndef DIGHOLO_B200_H
#define DIGHOLO_B200_H

#if defined(__cplusplus) && !defined(DIGHOLO_CXX_LINKAGE)
extern "C" {
#endif

typedef float complex64[2];               /* digHolo.h:163 */

/* error codes, digHolo.h:171-182 */
#define DIGHOLO_ERROR_SUCCESS 0
#define DIGHOLO_ERROR_ERROR 1
#define DIGHOLO_ERROR_INVALIDHANDLE 2
#define DIGHOLO_ERROR_NULLPOINTER 3
#define DIGHOLO_ERROR_SETFRAMEBUFFERDISABLED 4
#define DIGHOLO_ERROR_INVALIDDIMENSION 5
#define DIGHOLO_ERROR_INVALIDPOLARISATION 6
#define DIGHOLO_ERROR_INVALIDAXIS 7
#define DIGHOLO_ERROR_INVALIDARGUMENT 8
#define DIGHOLO_ERROR_MEMORYALLOCATION 9
#define DIGHOLO_ERROR_FILENOTCREATED 10
#define DIGHOLO_ERROR_FILENOTFOUND 11

/* averaging modes, digHolo.h:655-658 */
#define DIGHOLO_AVGMODE_SEQUENTIAL 0
#define DIGHOLO_AVGMODE_INTERLACED 1
#define DIGHOLO_AVGMODE_SEQUENTIALSWEEP 2
#define DIGHOLO_AVGMODE_COUNT 3

/* AutoAlign modes, digHolo.h:925-928 */
#define DIGHOLO_AUTOALIGNMODE_FULL 0
#define DIGHOLO_AUTOALIGNMODE_TWEAK 1
#define DIGHOLO_AUTOALIGNMODE_ESTIMATE 2
#define DIGHOLO_AUTOALIGNMODE_COUNT 3

/* basis types, digHolo.h:1348-1350 */
#define DIGHOLO_BASISTYPE_HG 0
#define DIGHOLO_BASISTYPE_LG 1
#define DIGHOLO_BASISTYPE_CUSTOM 2

/* metrics, digHolo.h:1363-1372 */
#define DIGHOLO_METRIC_IL 0
#define DIGHOLO_METRIC_MDL 1
#define DIGHOLO_METRIC_DIAG 2
#define DIGHOLO_METRIC_SNRAVG 3
#define DIGHOLO_METRIC_DIAGBEST 4
#define DIGHOLO_METRIC_DIAGWORST 5
#define DIGHOLO_METRIC_SNRBEST 6
#define DIGHOLO_METRIC_SNRWORST 7
#define DIGHOLO_METRIC_SNRMG 8
#define DIGHOLO_METRIC_COUNT 9

/* batch-summary parameters, digHolo.h:1624-1631 */
#define DIGHOLO_ANALYSIS_TOTALPOWER 0
#define DIGHOLO_ANALYSIS_COMX 1
#define DIGHOLO_ANALYSIS_COMY 2
#define DIGHOLO_ANALYSIS_MAXABS 3
#define DIGHOLO_ANALYSIS_MAXABSIDX 4
#define DIGHOLO_ANALYSIS_AEFF 5
#define DIGHOLO_ANALYSIS_COMYWRAP 6
#define DIGHOLO_ANALYSIS_COUNT 7

/* verbosity, digHolo.h:1906-1909 */
#define DIGHOLO_VERBOSITY_OFF 0
#define DIGHOLO_VERBOSITY_BASIC 1
#define DIGHOLO_VERBOSITY_DEBUG 2
#define DIGHOLO_VERBOSITY_COOKED 3

/* replaces digHolo.h:209 */
int digHoloCreate();
/* replaces digHolo.h:216 */
int digHoloDestroy(int handleIdx);
/* replaces digHolo.h:245 */
int digHoloSetFrameBuffer(int handleIdx, float* buffer);
/* replaces digHolo.h:255 */
float* digHoloGetFrameBuffer(int handleIdx);
/* replaces digHolo.h:268 */
int digHoloSetFrameBufferUint16(int handleIdx, unsigned short* buffer, int transposeMode);
/* replaces digHolo.h:277 */
unsigned short* digHoloGetFrameBufferUint16(int handleIdx, int* transposeMode);
/* replaces digHolo.h:298 */
int digHoloConfigSetFrameDimensions(int handleIdx, int width, int height);
/* replaces digHolo.h:308 */
int digHoloConfigGetFrameDimensions(int handleIdx, int* width, int* height);
/* replaces digHolo.h:317 */
int digHoloConfigSetFramePixelSize(int handleIdx, float pixelSize);
/* replaces digHolo.h:325 */
float digHoloConfigGetFramePixelSize(int handleIdx);
/* replaces digHolo.h:334 */
int digHoloConfigSetPolCount(int handleIdx, int polCount);
/* replaces digHolo.h:344 */
int digHoloConfigGetPolCount(int handleIdx);
/* replaces digHolo.h:449 */
int digHoloConfigSetFillFactorCorrectionEnabled(int handleIdx, int enabled);
/* replaces digHolo.h:460 */
int digHoloConfigGetFillFactorCorrectionEnabled(int handleIdx);
/* replaces digHolo.h:483 */
int digHoloSetBatch(int handleIdx, int batchCount, float* frameBuffer);
/* replaces digHolo.h:502 */
int digHoloSetBatchAvg(int handleIdx, int batchCount, float* frameBuffer, int avgCount, int avgMode);
/* replaces digHolo.h:519 */
int digHoloSetBatchUint16(int handleIdx, int batchCount, unsigned short* frameBuffer, int transpose);
/* replaces digHolo.h:540 */
int digHoloSetBatchAvgUint16(int handleIdx, int batchCount, unsigned short* frameBuffer, int avgCount, int avgMode, int transpose);
/* replaces digHolo.h:551 */
int digHoloConfigSetBatchCount(int handleIdx, int batchCount);
/* replaces digHolo.h:559 */
int digHoloConfigGetBatchCount(int handleIdx);
/* replaces digHolo.h:570 */
int digHoloConfigSetBatchAvgCount(int handleIdx, int avgCount);
/* replaces digHolo.h:580 */
int digHoloConfigGetBatchAvgCount(int handleIdx);
/* replaces digHolo.h:599 */
int digHoloConfigSetBatchCalibration(int handleIdx, complex64* cal, int polCount, int batchCount);
/* replaces digHolo.h:611 */
complex64* digHoloConfigGetBatchCalibration(int handleIdx, int *polCount, int *batchCount);
/* replaces digHolo.h:635 */
int digHoloConfigSetBatchCalibrationEnabled(int handleIdx, int enabled);
/* replaces digHolo.h:645 */
int digHoloConfigGetBatchCalibrationEnabled(int handleIdx);
/* replaces digHolo.h:670 */
int digHoloConfigSetBatchAvgMode(int handleIdx, int avgMode);
/* replaces digHolo.h:680 */
int digHoloConfigGetBatchAvgMode(int handleIdx);
/* replaces digHolo.h:701 */
int digHoloConfigSetfftWindowSize(int handleIdx, int width, int height);
/* replaces digHolo.h:712 */
int digHoloConfigGetfftWindowSize(int handleIdx, int *width, int *height);
/* replaces digHolo.h:722 */
int digHoloConfigSetfftWindowSizeX(int handleIdx, int width);
/* replaces digHolo.h:730 */
int digHoloConfigGetfftWindowSizeX(int handleIdx);
/* replaces digHolo.h:739 */
int digHoloConfigGetfftWindowSizeY(int handleIdx);
/* replaces digHolo.h:749 */
int digHoloConfigSetfftWindowSizeY(int handleIdx, int height);
/* replaces digHolo.h:766 */
int digHoloConfigSetFourierWindowRadius(int handleIdx, float windowRadius);
/* replaces digHolo.h:774 */
float digHoloConfigGetFourierWindowRadius(int handleIdx);
/* replaces digHolo.h:786 */
int digHoloConfigSetIFFTResolutionMode(int handleIdx, int resolutionModeIdx);
/* replaces digHolo.h:797 */
int digHoloConfigGetIFFTResolutionMode(int handleIdx);
/* replaces digHolo.h:814 */
int digHoloConfigSetWavelengthCentre(int handleIdx, float lambda0);
/* replaces digHolo.h:822 */
float digHoloConfigGetWavelengthCentre(int handleIdx);
/* replaces digHolo.h:938 */
int digHoloConfigSetAutoAlignBeamCentre(int handleIdx, int enable);
/* replaces digHolo.h:946 */
int digHoloConfigGetAutoAlignBeamCentre(int handleIdx);
/* replaces digHolo.h:955 */
int digHoloConfigSetAutoAlignDefocus(int handleIdx, int enable);
/* replaces digHolo.h:963 */
int digHoloConfigGetAutoAlignDefocus(int handleIdx);
/* replaces digHolo.h:972 */
int digHoloConfigSetAutoAlignTilt(int handleIdx, int enable);
/* replaces digHolo.h:980 */
int digHoloConfigGetAutoAlignTilt(int handleIdx);
/* replaces digHolo.h:989 */
int digHoloConfigSetAutoAlignBasisWaist(int handleIdx, int enable);
/* replaces digHolo.h:997 */
int digHoloConfigGetAutoAlignBasisWaist(int handleIdx);
/* replaces digHolo.h:1008 */
int digHoloConfigSetAutoAlignFourierWindowRadius(int handleIdx, int enable);
/* replaces digHolo.h:1016 */
int digHoloConfigGetAutoAlignFourierWindowRadius(int handleIdx);
/* replaces digHolo.h:1025 */
int digHoloConfigSetAutoAlignTol(int handleIdx, float tolerance);
/* replaces digHolo.h:1033 */
float digHoloConfigGetAutoAlignTol(int handleIdx);
/* replaces digHolo.h:1046 */
int digHoloConfigSetAutoAlignPolIndependence(int handleIdx, int polIndependence);
/* replaces digHolo.h:1058 */
int digHoloConfigGetAutoAlignPolIndependence(int handleIdx);
/* replaces digHolo.h:1071 */
int digHoloConfigSetAutoAlignBasisMulConjTrans(int handleIdx, int mulConjTranspose);
/* replaces digHolo.h:1083 */
int digHoloConfigGetAutoAlignBasisMulConjTrans(int handleIdx);
/* replaces digHolo.h:1101 */
int digHoloConfigSetAutoAlignMode(int handleIdx, int alignMode);
/* replaces digHolo.h:1109 */
int digHoloConfigGetAutoAlignMode(int handleIdx);
/* replaces digHolo.h:1128 */
int digHoloConfigSetAutoAlignGoalIdx(int handleIdx, int goalIdx);
/* replaces digHolo.h:1136 */
int digHoloConfigGetAutoAlignGoalIdx(int handleIdx);
/* replaces digHolo.h:1152.  The reference's AutoAlign with every
 * evaluation on the GPU, returning the final value of the goal metric in dB:
 * FULL (the default) and ESTIMATE first run the parameter estimate from the
 * full Fourier planes (tilt by the DCT correlation of the batch-summed
 * Fourier intensity, window radius, waist from the effective areas, beam
 * centre from the camera-plane centre of mass, defocus by the focus search;
 * digHolo.cpp:11517-11970, 11181-11499); FULL and TWEAK then run the
 * coordinate search (tilt, beam centre, defocus, waist; optional
 * Fourier-window radius rule), with a second pass on the goal when the goal
 * is not IL. */
float digHoloAutoAlign(int handleIdx);
/* replaces digHolo.h:1163 */
float digHoloAutoAlignGetMetric(int handleIdx, int metricIdx);
/* replaces digHolo.h:1174 */
float* digHoloAutoAlignGetMetrics(int handleIdx, int metricIdx);
/* replaces digHolo.h:1185.  IL, MDL (FP64 Gram eigenvalues on the GPU),
 * SNR, diagonal/crosstalk metrics of the last processed batch. */
int digHoloAutoAlignCalcMetrics(int handleIdx);
/* replaces digHolo.h:1205 */
int digHoloConfigSetBeamCentre(int handleIdx, int axisIdx, int polIdx, float centre);
/* replaces digHolo.h:1215 */
float digHoloConfigGetBeamCentre(int handleIdx, int axisIdx, int polIdx);
/* replaces digHolo.h:1226 */
int digHoloConfigSetTilt(int handleIdx, int axisIdx, int polIdx, float tilt);
/* replaces digHolo.h:1236 */
float digHoloConfigGetTilt(int handleIdx, int axisIdx, int polIdx);
/* replaces digHolo.h:1246 */
int digHoloConfigSetDefocus(int handleIdx, int polIdx, float defocus);
/* replaces digHolo.h:1255 */
float digHoloConfigGetDefocus(int handleIdx, int polIdx);
/* replaces digHolo.h:1270 */
int digHoloConfigSetPolLockTilt(int handleIdx, int polLock);
/* replaces digHolo.h:1282 */
int digHoloConfigGetPolLockTilt(int handleIdx);
/* replaces digHolo.h:1297 */
int digHoloConfigSetPolLockDefocus(int handleIdx, int polLock);
/* replaces digHolo.h:1309 */
int digHoloConfigGetPolLockDefocus(int handleIdx);
/* replaces digHolo.h:1318 */
int digHoloConfigSetPolLockBasisWaist(int handleIdx, int polLock);
/* replaces digHolo.h:1326 */
int digHoloConfigGetPolLockBasisWaist(int handleIdx);
/* replaces digHolo.h:1384 */
int digHoloConfigSetBasisGroupCount(int handleIdx, int groupCount);
/* replaces digHolo.h:1393 */
int digHoloConfigGetBasisGroupCount(int handleIdx);
/* replaces digHolo.h:1404 */
int digHoloConfigSetBasisWaist(int handleIdx, int polIdx, float waist);
/* replaces digHolo.h:1416 */
float digHoloConfigGetBasisWaist(int handleIdx, int polIdx);
/* replaces digHolo.h:1424 */
int digHoloConfigSetBasisTypeHG(int handleIdx);
/* replaces digHolo.h:1435: coefficients returned in the Laguerre-Gaussian basis */
int digHoloConfigSetBasisTypeLG(int handleIdx);
/* replaces digHolo.h:1453: coefficients returned in a custom basis; transform is
 * [modeCountIn][modeCountOut] complex (copied), HG mode i onto custom mode j */
int digHoloConfigSetBasisTypeCustom(int handleIdx, int modeCountIn, int modeCountOut, complex64* transform);
/* replaces digHolo.h:1464: returns the type set (0 HG, 1 LG, 2 custom) */
int digHoloConfigSetBasisType(int handleIdx, int basisType);
/* replaces digHolo.h:1472 */
int digHoloConfigGetBasisType(int handleIdx);
/* replaces digHolo.h:1494 */
complex64* digHoloProcessBatch(int handleIdx, int* batchCount, int* modeCount, int* polCount);
/* replaces digHolo.h:1549 */
complex64* digHoloGetFields(int handleIdx, int* batchCount, int* polCount, float** x, float** y, int* width, int* height);
/* replaces digHolo.h:1568 */
int digHoloGetFields16(int handleIdx, int* batchCount, int* polCount, short** fieldR, short** fieldI, float** fieldScale, float** x, float** y, int* width, int* height);
/* replaces digHolo.h:1603 */
complex64* digHoloBasisGetCoefs(int handleIdx, int* batchCount, int* modeCount, int* polCount);
/* replaces digHolo.h:1659 */
int digHoloBatchGetSummary(int handleIdx, int planeIdx, int* parameterCount, int* totalCount, int* polCount, float** parameters, int* pixelCountX, int* pixelCountY, float** xAxis, float** yAxis, float** totalIntensity);
/* replaces digHolo.h:1670 */
int digHoloProcessFFT(int handleIdx);
/* replaces digHolo.h:1682 */
int digHoloProcessIFFT(int handleIdx);
/* replaces digHolo.h:1694 */
int digHoloProcessRemoveTilt(int handleIdx);
/* replaces digHolo.h:1706 */
int digHoloProcessBasisExtractCoefs(int handleIdx);
/* replaces digHolo.h:1718.  The R2C Fourier planes [batch][pol][H][W/2+1]
 * of the last batch, computed from its frames on the first call after the
 * batch (the frame buffer must still be valid, as for ProcessBatch); *width
 * is the FFT window width W, as in the reference. */
complex64* digHoloGetFourierPlaneFull(int handleIdx, int* batchCount, int* polCount, int* width, int* height);
/* replaces digHolo.h:1732 */
complex64* digHoloGetFourierPlaneWindow(int handleIdx, int* batchCount, int* polCount, int* width, int* height);
/* replaces digHolo.h:1776.  Batches per second over about goalDuration
 * seconds of digHoloProcessBatch; info[6] (optional) per-stage rates
 * (DIGHOLO_BENCHMARK_FFT .. TOTAL, digHolo.h:1783-1788). */
float digHoloBenchmark(int handleIdx, float goalDuration, float* info);
/* replaces digHolo.h:1749 */
int digHoloConfigSetThreadCount(int handleIdx, int threadCount);
/* replaces digHolo.h:1757 */
int digHoloConfigGetThreadCount(int handleIdx);
/* replaces digHolo.h:1808 */
int digHoloConfigSetFFTWPlanMode(int handleIdx, int planningMode);
/* replaces digHolo.h:1818 */
int digHoloConfigGetFFTWPlanMode(int handleIdx);
/* replaces digHolo.h:1825: forgets the tuned kernel plans (the wisdom of
 * plan modes 1-3), not the wisdom file */
int digHoloFFTWWisdomForget();
/* replaces digHolo.h:1835: the file the tuned kernel plans are loaded from
 * (before the next lookup) and saved to (after every new plan) */
int digHoloFFTWWisdomFilename(const char* filename);
/* replaces digHolo.h:1924 */
int digHoloConfigSetVerbosity(int handleIdx, int verbosity);
/* replaces digHolo.h:1937 */
int digHoloConfigGetVerbosity(int handleIdx);
/* replace digHolo.h:832, 843, 854, 886, 895: the wavelengths of the frames
 * of a batch (taking effect at the next processing), as an array or equally
 * spaced in frequency; an array of one wavelength means the centre
 * wavelength; the ordering of frames (inoutIdx 0) and outputs (1): 0
 * wavelength the fast axis, 1 the slow axis */
int digHoloConfigSetWavelengths(int handleIdx, float* wavelengths, int wavelengthCount);
int digHoloConfigSetWavelengthsLinearFrequency(int handleIdx, float wavelengthStart, float wavelengthStop,
                                               int wavelengthCount);
float* digHoloConfigGetWavelengths(int handleIdx, int* wavelengthCount);
int digHoloConfigSetWavelengthOrdering(int handleIdx, int inoutIdx, int ordering);
int digHoloConfigGetWavelengthOrdering(int handleIdx, int inoutIdx);
/* replace digHolo.h:1510 and 1525: ProcessBatch of frames at several
 * wavelengths; each wavelength's frames run as one sub-batch with its own
 * Fourier-window mask and reference wave in the common IFFT window; the
 * batch count must be a multiple of the wavelength count, without frame
 * averaging */
complex64* digHoloProcessBatchFrequencySweepLinear(int handleIdx, int* batchCount, int* modeCount, int* polCount,
                                                   float lambdaStart, float lambdaStop, int lambdaCount);
complex64* digHoloProcessBatchWavelengthSweepArbitrary(int handleIdx, int* batchCount, int* modeCount, int* polCount,
                                                       float* wavelengths, int lambdaCount);
/* replace digHolo.h:369, 384, 400, 409, 417, 437: the reference-wave
 * calibration, stored as the reference normalises and inverts it; while
 * enabled and of the frames' size, its reconstructed planes (c2c FFT of the
 * FFT windows, Fourier window at zero tilt, IFFT; digHolo.cpp:6729-6830,
 * 8253-8285) multiply every frame's IFFT output before the field analysis
 * (digHolo.cpp:8736-8758).
 * GetRefCalibrationFields returns the planes [item][pol][height][width] for
 * the last batch's geometry, NULL before one. */
int digHoloConfigSetRefCalibrationIntensity(int handleIdx, unsigned short* cal, int wavelengthCount, int width,
                                            int height);
int digHoloConfigSetRefCalibrationField(int handleIdx, complex64* cal, int wavelengthCount, int width, int height);
int digHoloConfigSetRefCalibrationFromFile(int handleIdx, const char* fname, int wavelengthCount, int width,
                                           int height);
int digHoloConfigSetRefCalibrationEnabled(int handleIdx, int enabled);
int digHoloConfigGetRefCalibrationEnabled(int handleIdx);
complex64* digHoloConfigGetRefCalibrationFields(int handleIdx, int* wavelengthCount, int* polCount, float** x,
                                                float** y, int* width, int* height);
/* replaces digHolo.h:1962: one batch described by a settings file (tab-
 * separated names and values, the reference's names), its outputs written
 * to the files the settings name; digholo_b200/digholo_run runs it for each
 * file named on its command line */
int digHoloRunBatchFromConfigFile(char* filename);
/* replaces digHolo.h:288: uint16 frames from a binary file, held by the
 * handle (as float32) as its frame buffer */
int digHoloSetFrameBufferFromFile(int handleIdx, const char* fname);
/* replaces digHolo.h:624: polCount x batchCount complex64 from a file */
int digHoloConfigSetBatchCalibrationFromFile(int handleIdx, const char* fname, int polCount, int batchCount);
/* replaces digHolo.h:1587: the basis fields of the last batch's basis,
 * modeCount x polCount x height x width complex64 (computed on the GPU) */
complex64* digHoloBasisGetFields(int handleIdx, int* modeCount, int* polCount, float** x, float** y, int* width,
                                 int* height);
/* replaces digHolo.h:1766: the configured thread count (the GPU path has
 * no CPU thread pool to tune) */
int digHoloBenchmarkEstimateThreadCountOptimal(int handleIdx, float goalDuration);
/* replace digHolo.h:1883 and 1897: the viewport bitmap renderer is not part
 * of this library; no bitmap, zero width and height, DIGHOLO_ERROR_ERROR */
unsigned char* digHoloGetViewport(int handleIdx, int displayMode, int forceProcessing, int* width, int* height,
                                  char** windowString);
int digHoloGetViewportToFile(int handleIdx, int displayMode, int forceProcessing, int* width, int* height,
                             char** windowString, const char* filename);
/* replace digHolo.h:1945 and 1952 */
int digHoloConsoleRedirectToFile(char* filename);
int digHoloConsoleRestore();
/* replace digHolo.h:1973 and 1983 */
int digHoloConfigBackupSave(int handleIdx);
int digHoloConfigBackupLoad(int handleIdx);
/* replaces digHolo.h:1990 (not for general use; does nothing here) */
void digHoloDebugRoutine(int handleIdx);
/* replace digHolo.h:2075 and 2084: rows of six Zernike coefficients per
 * polarisation (tilt x, tilt y at 1, 2; defocus at 4) */
float** digHoloConfigGetZernCoefs(int handleIdx);
int digHoloConfigGetZernCount(int handleIdx);
/* replaces digHolo.h:2026: synthetic camera frames, computed on the GPU,
 * returned in one host allocation ([float32 frames][uint16 frames]
 * [parameters]) released by digHoloFrameSimulatorDestroy; null arrays take
 * the reference's defaults and are pointed at them; wavelengthOrdering is
 * accepted (the reference's frames do not depend on it) */
float* digHoloFrameSimulatorCreate(int frameCount, int* frameWidth, int* frameHeight, float* pixelSize, int* polCount,
                                   float** refTiltX, float** refTiltY, float** refDefocus, float** refWaist,
                                   float** refBeamCentreX, float** refBeamCentreY, complex64** refAmplitude,
                                   int* beamGroupCount, float** beamWaist, complex64** beamCoefs, float** beamCentreX,
                                   float** beamCentreY, int* cameraPixelLevelCount, int fillFactorCorrection,
                                   float** wavelengths, int* wavelengthCount, int wavelengthOrdering, int printToConsole,
                                   unsigned short** pixelBuffer16, const char* fname);
/* replaces digHolo.h:2046 */
float* digHoloFrameSimulatorCreateSimple(int frameCount, int frameWidth, int frameHeight, float pixelSize, int polCount,
                                         float wavelength, int printToConsole);
/* replaces digHolo.h:2056 */
int digHoloFrameSimulatorDestroy(float* pixelBuffer);

/* ------------------------------------------------------------------------
 * Extensions with no counterpart in the reference.
 * ---------------------------------------------------------------------- */

/* Runs the batch path on frames already in device memory (digHoloSetBatch*
 * given a device pointer) and leaves every output on the device; returns
 * without waiting for the GPU. */
int digHoloB200ProcessBatchDevice(int handleIdx);

/* Device pointer to the coefficients [batch][pol * mode] of the last batch. */
complex64* digHoloB200GetCoefsDevice(int handleIdx, int* batchCount, int* modeCount, int* polCount);

/* Waits for the handle's GPU work (DIGHOLO_ERROR_ERROR on a CUDA error). */
int digHoloB200Synchronize(int handleIdx);

/* Runs the handle's GPU work on a caller-owned cudaStream_t (nullptr: a
 * private stream).  Call before the first processing. */
int digHoloB200SetStream(int handleIdx, void* stream);

/* Keep the float field -conj(A.ref) computed with the unquantised reference
 * wave, next to the int16 field; read it with digHoloB200GetFields32. */
int digHoloB200SetKeepField32(int handleIdx, int enable);
complex64* digHoloB200GetFields32(int handleIdx, int* batchCount, int* polCount, int* width, int* height);

/* CUDA-event timing of the forward and inverse kernels: out3 = {forward ms
 * summed, inverse ms summed, batches} since the previous call. */
int digHoloB200SetTiming(int handleIdx, int enable);
int digHoloB200GetStageTimes(int handleIdx, float* out3);

/* Batches on device-resident frames replay their forward and inverse
 * launches from a CUDA graph once the same launch arguments recur (on by
 * default; the first batch with new arguments runs directly, the second is
 * captured).  0 launches directly and releases the graphs.  GetGraphCount:
 * graphs held (at most 8). */
int digHoloB200SetGraphs(int handleIdx, int enable);
int digHoloB200GetGraphCount(int handleIdx);

/* Window geometry of the last batch: W, H, w, h, nx, ny, FFT-window corner
 * (x, y) and IFFT-window origin (SX, SY) of polarisation 0. */
int digHoloB200GetGeometry(int handleIdx, int* out10);

/* Forward kernel choice (testing aid): 0 automatic (for uint16 frames the
 * tensor-core row-DFT kernel, else the TMA-fed persistent kernel where shape
 * and alignment allow, else the register kernel, else the generic one),
 * 1 generic shared-memory kernel, 2 register kernel, 3 TMA-fed kernel only,
 * 4 tensor-core row-DFT kernel only (uint16 frames, 128-row FFT windows 64
 * or 128 wide, 16- or 32-pixel IFFT windows), 5 R2C planes (rows, then
 * columns, then the window; automatic for windows 256 pixels wide or more;
 * 512-pixel rows by a register transform and, for 64-row IFFT windows, only
 * the window's columns and rows computed);
 * the batch fails where the chosen kernel does not apply. */
int digHoloB200SetForwardKernel(int handleIdx, int kernel);
/* Forward kernel the last batch ran: 1 generic, 2 register, 3 TMA-fed,
 * 4 tensor-core row DFT, 5 full planes. */
int digHoloB200GetForwardKernel(int handleIdx);
/* Inverse kernel choice (testing aid): 0 automatic (one warp per frame and
 * polarisation for 16- and 32-pixel low-resolution fields; for
 * full-resolution fields the pruned field kernel followed by the overlap
 * kernel up to 128 x 128 pixels, bands of 64 rows beyond; else one block),
 * 1 one block per frame and polarisation, 2 full-resolution bands only (the
 * batch fails where they do not apply: low resolution, fields under 64 x 64,
 * windows under 16 pixels; beyond 32 mode groups the bands write the fields
 * and the chunked FP32 overlap follows), 3 as 0 but fused into the
 * tensor-core forward kernel where it applies (uint16 frames, 16 x 16
 * low-resolution fields: one launch per batch). */
int digHoloB200SetInverseKernel(int handleIdx, int kernel);
/* Inverse kernel the last batch ran: 1 block per unit, 2 low-resolution
 * 16/32-pixel fields (64 threads / one warp per unit), 3 full-resolution
 * field kernel + overlap kernel, 4 full-resolution bands (statistics pass,
 * quantising pass with the overlap, coefficient sum), 5 fused into the
 * tensor-core forward kernel (inverse choice 3), 6 low-resolution fields
 * whose sides are multiples of 16 but not powers of two (direct DFT),
 * 7 full-resolution 64-point bands (512-wide fields, IFFT windows up to
 * 64 x 64). */
int digHoloB200GetInverseKernel(int handleIdx);
/* Overlap of full-resolution fields: 0 (default) on the tensor cores in
 * split-BF16 precision (bf16 hi + lo of both int16 operands, three products,
 * FP32 accumulation) where the field shape allows, 1 FP32 on the CUDA cores. */
int digHoloB200SetOverlapKernel(int handleIdx, int kernel);
/* Overlap the last batch ran: 1 FP32 CUDA cores, 2 split-BF16 tensor cores. */
int digHoloB200GetOverlapKernel(int handleIdx);

/* Message of the handle's last error ("" when none). */
const char* digHoloB200GetLastError(int handleIdx);

/* Gradient of IL = 10 log10(sum |c|^2) + const with respect to
 * grad12[pol * 6 + k], k = tiltX (deg), tiltY (deg), defocus, beamCentreX (m),
 * beamCentreY (m), waist (m), at the current configuration with the
 * Fourier-window selection held fixed: one batch pass and its adjoint on the
 * GPU.  Parameters tied by the polarisation locks carry the sum on
 * polarisation 0.  *il (optional) = 10 log10(sum |c|^2). */
int digHoloB200AutoAlignGradient(int handleIdx, float* grad12, float* il);
/* The same for metricIdx DIGHOLO_METRIC_IL (0) or DIGHOLO_METRIC_MDL (1):
 * MDL = 10 log10(s_min^2 / s_max^2) of the batch coefficient matrix (the
 * power meter's blocks: both polarisations together, or each alone with
 * AutoAlignPolIndependence), its gradient through the derivatives of the
 * extreme eigenvalues of the FP64 Gram matrix, d lambda = u^H dG u.
 * *value (optional) = the metric in dB.  No counterpart in the reference. */
int digHoloB200AutoAlignGradientMetric(int handleIdx, int metricIdx, float* grad12, float* value);
/* 1: hold the FFT window and the Fourier-window selection and mask at the
 * current settings (the beam-centre phase, reference wave and basis keep
 * following the configuration), as the gradient assumes; 0: release. */
int digHoloB200FreezeWindow(int handleIdx, int enable);
/* Gradient-driven AutoAlign (goal IL): quasi-Newton (BFGS) on the adjoint
 * gradient over the enabled alignment parameters.  Returns the goal metric
 * of the final configuration; digHoloAutoAlignGetMetric(s) read the metrics. */
float digHoloB200AutoAlignAdjoint(int handleIdx);

/* Number of batch evaluations (window selection, tilt removal, overlap and
 * power meter) the last digHoloAutoAlign call made. */
int digHoloB200GetAutoAlignEvaluations(int handleIdx);

/* No counterpart in the reference.  The kernel plan tuned for the handle's
 * current shape (plan modes 1-3, see digHoloConfigSetFFTWPlanMode): returns 1
 * and the forward / inverse kernel choices (as digHoloB200SetForwardKernel /
 * SetInverseKernel number them) and the batch time in ms, or 0 when the shape
 * has no plan.  digHoloB200GetKernelPlanRuns: tuning runs in this process. */
int digHoloB200GetKernelPlan(int handleIdx, int* forwardKernel, int* inverseKernel, float* ms);
int digHoloB200GetKernelPlanRuns();

/* No counterpart in the reference (its power meter calls LAPACK cgesvd).
 * Eigenvalues of one Hermitian n x n matrix, FP64, with the GPU solver
 * behind MDL: G (host) column-major complex double (re, im interleaved),
 * W (host) n eigenvalues ascending; with vecs non-null (host, 2 n complex
 * double) the unit eigenvectors of the smallest and the largest eigenvalue.
 * n up to 2048.  Runs on the current device and waits for it. */
int digHoloB200EigenHermitian(int n, const double* G, double* W, double* vecs);

/* No counterpart in the reference.  digHoloFrameSimulatorCreate with the
 * frames left in device memory: the same parameters by value (null arrays
 * take the same defaults; frame sides must be multiples of 16), frames32 a
 * device buffer of frameCount x frameHeight x frameWidth float32 (required:
 * the intensities are formed there), frames16 an optional device uint16
 * buffer of the same shape.  Returns a DIGHOLO_ERROR code. */
int digHoloB200FrameSimulatorDevice(int frameCount, int frameWidth, int frameHeight, float pixelSize, int polCount,
                                    const float* refTiltX, const float* refTiltY, const float* refDefocus,
                                    const float* refWaist, const float* refBeamCentreX, const float* refBeamCentreY,
                                    int beamGroupCount, const float* beamWaist, const complex64* beamCoefs,
                                    const float* beamCentreX, const float* beamCentreY, int cameraPixelLevelCount,
                                    int fillFactorCorrection, const float* wavelengths, int wavelengthCount,
                                    float* frames32, unsigned short* frames16);

/* No counterpart in the reference.  The batch path for callers that cannot
 * allocate device memory while they process frames (a real-time acquisition
 * callback must not block in cudaMalloc/cudaFree, which can synchronise the
 * device; some applications fix their memory pool at start-up).  Nothing is
 * allocated: the scratch carrying the Fourier windows between the two
 * kernels is a static 8 MiB device array, and the caller passes the device
 * frames and device outputs -- coefs [frame][pol*mode] complex64, fieldR and
 * fieldI [frame][pol][ny][nx] int16, stats [7][pol][frameCount+1] float (the
 * aggregate column is not written).  The handle must already hold the tables
 * for its configuration (process one batch with digHoloProcessBatch or
 * digHoloB200ProcessBatchDevice first; that call allocates).  Sizes with
 * frameCount*polCount*w*h*8 bytes above 8 MiB are refused with
 * DIGHOLO_ERROR_INVALIDDIMENSION.  Where the preparing batch sized a scratch
 * of the handle (the Fourier planes of windows 256 pixels wide and more, the
 * band buffers of large full-resolution fields), a frameCount above that
 * batch's is refused with DIGHOLO_ERROR_MEMORYALLOCATION, not allocated.
 * The call makes the handle's device current and leaves it so; the first
 * call on a device looks up the scratch address there
 * (cudaGetSymbolAddress; with CUDA's lazy module loading the 8 MiB array is
 * placed in device memory at that moment): make it before any stream capture.
 * Calls share the scratch; calls whose GPU work overlaps race on it.
 * Returns without waiting for the GPU (see digHoloB200Synchronize). */
int digHoloB200ProcessBatchNoAlloc(int handleIdx, const void* frames, int frameCount, int framesAreUint16,
                                   complex64* coefs, short* fieldR, short* fieldI, float* stats);

#if defined(__cplusplus) && !defined(DIGHOLO_CXX_LINKAGE)
}
#endif

#endif /* DIGHOLO_B200_H */
