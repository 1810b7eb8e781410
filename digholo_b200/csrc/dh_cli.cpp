// digHoloRunBatchFromConfigFile (digHolo.h:1962, digHolo.cpp:16766-17931):
// run one batch described by a settings file through this library's
// entry points, and the command-line runner around it (dh_cli_main.cpp,
// built as digholo_b200/digholo_run; the reference's main,
// digHolo.cpp:17934-17943).
//
// The settings file has one setting per line: its name, then its values,
// separated by tabs (digHolo.cpp:16829-16850).  The names, their effect and
// the order of the work after reading follow the reference: frame source (a
// uint16 file, or simulated frames when FrameBufferFilename has no value),
// configuration, wavelength sweep, reference and batch calibrations, custom
// basis, AutoAlign when any AutoAlign* switch is set, benchmark, the batch,
// then the output files (coefficients, basis fields, fields: complex64
// binary; x and y axes: float32 binary) and the text summary
// (digHolo.cpp:17336-17900).  The viewport names are accepted; this library
// has no viewport renderer, so no bitmaps are written.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

typedef float complex64[2];

extern "C" {
int digHoloCreate();
int digHoloDestroy(int h);
int dhHandleCount();
int digHoloSetFrameBufferFromFile(int h, const char* fname);
int digHoloConfigSetFrameDimensions(int h, int width, int height);
int digHoloConfigGetFrameDimensions(int h, int* width, int* height);
int digHoloConfigSetBatchCount(int h, int batchCount);
int digHoloConfigGetBatchCount(int h);
int digHoloConfigSetPolCount(int h, int polCount);
int digHoloConfigGetPolCount(int h);
int digHoloConfigSetVerbosity(int h, int verbosity);
int digHoloConfigSetThreadCount(int h, int threadCount);
int digHoloConfigSetFourierWindowRadius(int h, float radius);
float digHoloConfigGetFourierWindowRadius(int h);
int digHoloConfigSetBeamCentre(int h, int axisIdx, int polIdx, float value);
float digHoloConfigGetBeamCentre(int h, int axisIdx, int polIdx);
int digHoloConfigSetTilt(int h, int axisIdx, int polIdx, float value);
float digHoloConfigGetTilt(int h, int axisIdx, int polIdx);
int digHoloConfigSetDefocus(int h, int polIdx, float value);
float digHoloConfigGetDefocus(int h, int polIdx);
int digHoloConfigSetFramePixelSize(int h, float pixelSize);
float digHoloConfigGetFramePixelSize(int h);
int digHoloConfigSetPolLockTilt(int h, int v);
int digHoloConfigSetPolLockDefocus(int h, int v);
int digHoloConfigSetPolLockBasisWaist(int h, int v);
int digHoloConfigSetfftWindowSizeX(int h, int v);
int digHoloConfigSetfftWindowSizeY(int h, int v);
int digHoloConfigSetFFTWPlanMode(int h, int v);
int digHoloFFTWWisdomFilename(const char* filename);
int digHoloConfigSetIFFTResolutionMode(int h, int v);
int digHoloConfigSetWavelengthCentre(int h, float v);
int digHoloConfigSetWavelengthOrdering(int h, int inoutIdx, int ordering);
int digHoloConfigGetWavelengthOrdering(int h, int inoutIdx);
int digHoloConfigSetWavelengthsLinearFrequency(int h, float start, float stop, int count);
float* digHoloConfigGetWavelengths(int h, int* count);
int digHoloConfigSetBasisGroupCount(int h, int v);
int digHoloConfigGetBasisGroupCount(int h);
int digHoloConfigSetBasisType(int h, int v);
int digHoloConfigGetBasisType(int h);
int digHoloConfigSetBasisTypeCustom(int h, int modeCountIn, int modeCountOut, complex64* transform);
int digHoloConfigSetBasisWaist(int h, int polIdx, float v);
float digHoloConfigGetBasisWaist(int h, int polIdx);
int digHoloConfigSetBatchAvgCount(int h, int v);
int digHoloConfigGetBatchAvgCount(int h);
int digHoloConfigSetBatchAvgMode(int h, int v);
int digHoloConfigGetBatchAvgMode(int h);
int digHoloConfigSetAutoAlignBeamCentre(int h, int v);
int digHoloConfigSetAutoAlignDefocus(int h, int v);
int digHoloConfigSetAutoAlignTilt(int h, int v);
int digHoloConfigSetAutoAlignBasisWaist(int h, int v);
int digHoloConfigSetAutoAlignFourierWindowRadius(int h, int v);
int digHoloConfigSetAutoAlignTol(int h, float v);
int digHoloConfigSetAutoAlignPolIndependence(int h, int v);
int digHoloConfigSetAutoAlignBasisMulConjTrans(int h, int v);
int digHoloConfigSetAutoAlignMode(int h, int v);
int digHoloConfigSetAutoAlignGoalIdx(int h, int v);
int digHoloConfigSetFillFactorCorrectionEnabled(int h, int v);
int digHoloConfigGetFillFactorCorrectionEnabled(int h);
int digHoloConfigSetRefCalibrationFromFile(int h, const char* fname, int count, int width, int height);
complex64* digHoloConfigGetRefCalibrationFields(int h, int* count, int* polCount, float** x, float** y, int* w,
                                                int* hh);
int digHoloConfigSetBatchCalibrationFromFile(int h, const char* fname, int polCount, int batchCount);
int digHoloSetBatchAvg(int h, int batchCount, float* buffer, int avgCount, int avgMode);
float digHoloAutoAlign(int h);
float digHoloAutoAlignGetMetric(int h, int metricIdx);
int digHoloAutoAlignCalcMetrics(int h);
int digHoloBenchmarkEstimateThreadCountOptimal(int h, float goalDuration);
float digHoloBenchmark(int h, float goalDuration, float* info);
void digHoloDebugRoutine(int h);
complex64* digHoloProcessBatch(int h, int* batchCount, int* modeCount, int* polCount);
complex64* digHoloBasisGetFields(int h, int* modeCount, int* polCount, float** x, float** y, int* w, int* hh);
complex64* digHoloGetFields(int h, int* batchCount, int* polCount, float** x, float** y, int* w, int* hh);
int digHoloConsoleRedirectToFile(char* filename);
float* digHoloFrameSimulatorCreate(int frameCount, int* frameWidth, int* frameHeight, float* pixelSize, int* polCount,
                                   float** refTiltX, float** refTiltY, float** refDefocus, float** refWaist,
                                   float** refBeamCentreX, float** refBeamCentreY, float** refAmplitude,
                                   int* beamGroupCount, float** beamWaist, float** beamCoefs, float** beamCentreX,
                                   float** beamCentreY, int* cameraPixelLevelCount, int fillFactorCorrection,
                                   float** wavelengths, int* wavelengthCount, int wavelengthOrdering, int printToConsole,
                                   unsigned short** pixelBuffer16, const char* fname);
int digHoloFrameSimulatorDestroy(float* pixelBuffer);
}

namespace dh {
FILE* console();
}

namespace {

const int ERR_SUCCESS = 0, ERR_ERROR = 1, ERR_NULLPOINTER = 3, ERR_FILENOTFOUND = 11;
const int METRIC_IL = 0, METRIC_MDL = 1, METRIC_SNRAVG = 3;

// Settings gathered while reading, acted on afterwards.
struct Run {
    std::string consoleFile, outSummary, outCoefs, outFields, outBasis, outX, outY, outCalibration, outViewport;
    std::string basisFile, calibrationFile, batchCalibrationFile;
    int basisIn = 0, basisOut = 0;
    bool calibration = false, batchCalibration = false;
    int batchCalPol = 0, batchCalCount = 0;
    int autoAlign = 0, threadDiagnostic = 0, debug = 0, testFrames = 0;
    float benchmark = 0;
    std::vector<int> viewport;
    int wavelengthCount = 0;
    float wavelengthStart = 0, wavelengthStop = 0;
    bool tilt = false, centre = false, waist = false, defocus = false;
};

bool writeBinary(const std::string& name, const void* data, size_t elemBytes, size_t count) {
    FILE* f = fopen(name.c_str(), "wb");
    if (!f) return false;
    if (data && count) fwrite(data, elemBytes, count, f);
    fclose(f);
    return true;
}

// One setting line with values.  Returns false on a fatal error.
bool applySetting(int h, const std::string& name, const std::vector<std::string>& args, Run& run, int& errorCode) {
    const char* n = name.c_str();
    const size_t argc = args.size();
    auto is = [&](const char* key) { return !strcmp(key, n); };
    auto i0 = [&]() { return std::stoi(args[0]); };
    auto f0 = [&]() { return std::stof(args[0]); };
    if (is("FrameWidth")) {
        int w = 0, hh = 0;
        digHoloConfigGetFrameDimensions(h, &w, &hh);
        digHoloConfigSetFrameDimensions(h, i0(), hh);
    } else if (is("FrameHeight")) {
        int w = 0, hh = 0;
        digHoloConfigGetFrameDimensions(h, &w, &hh);
        digHoloConfigSetFrameDimensions(h, w, i0());
    } else if (is("BatchCount")) {
        digHoloConfigSetBatchCount(h, i0());
    } else if (is("PolCount")) {
        digHoloConfigSetPolCount(h, i0());
    } else if (is("ConsoleFilename")) {
        run.consoleFile = args[0];
    } else if (is("Verbosity")) {
        digHoloConfigSetVerbosity(h, i0());
    } else if (is("OutputFilenameSummary")) {
        run.outSummary = args[0];
    } else if (is("OutputFilenameCoefs")) {
        run.outCoefs = args[0];
    } else if (is("OutputFilenameFields")) {
        run.outFields = args[0];
    } else if (is("OutputFilenameBasis")) {
        run.outBasis = args[0];
    } else if (is("OutputFilenameXaxis")) {
        run.outX = args[0];
    } else if (is("OutputFilenameYaxis")) {
        run.outY = args[0];
    } else if (is("OutputFilenameRefCalibration")) {
        run.outCalibration = args[0];
    } else if (is("OutputFilenameViewport")) {
        run.outViewport = args[0];
    } else if (is("ThreadCount")) {
        const int v = i0();
        if (v <= 0) run.threadDiagnostic = 1;
        digHoloConfigSetThreadCount(h, v);
    } else if (is("Benchmark")) {
        run.benchmark = f0();
    } else if (is("Debug")) {
        run.debug = i0();
    } else if (is("FourierWindowRadius")) {
        digHoloConfigSetFourierWindowRadius(h, f0());
    } else if (is("BeamCentreX") || is("BeamCentreY") || is("TiltX") || is("TiltY")) {
        const int axis = (is("BeamCentreX") || is("TiltX")) ? 0 : 1;
        const bool centre = is("BeamCentreX") || is("BeamCentreY");
        for (size_t a = 0; a < argc; a++) {
            const float v = std::stof(args[a]);
            if (centre) {
                run.centre = run.centre || v != 0;
                digHoloConfigSetBeamCentre(h, axis, (int)a, v);
            } else {
                run.tilt = run.tilt || v != 0;
                digHoloConfigSetTilt(h, axis, (int)a, v);
            }
        }
    } else if (is("Defocus")) {
        for (size_t a = 0; a < argc; a++) {
            const float v = std::stof(args[a]);
            run.defocus = run.defocus || v != 0;
            digHoloConfigSetDefocus(h, (int)a, v);
        }
    } else if (is("PixelSize") || is("FramePixelSize")) {
        digHoloConfigSetFramePixelSize(h, f0());
    } else if (is("PolLockTilt")) {
        digHoloConfigSetPolLockTilt(h, i0());
    } else if (is("PolLockDefocus")) {
        digHoloConfigSetPolLockDefocus(h, i0());
    } else if (is("PolLockBasisWaist") || is("PolLockWaist")) {
        digHoloConfigSetPolLockBasisWaist(h, i0());
    } else if (is("fftWindowSizeX")) {
        digHoloConfigSetfftWindowSizeX(h, i0());
    } else if (is("fftWindowSizeY")) {
        digHoloConfigSetfftWindowSizeY(h, i0());
    } else if (is("FFTWPlanMode")) {
        digHoloConfigSetFFTWPlanMode(h, i0());
    } else if (is("FFTWWisdomFilename")) {
        digHoloFFTWWisdomFilename(args[0].c_str());
    } else if (is("IFFTResolutionMode")) {
        digHoloConfigSetIFFTResolutionMode(h, i0());
    } else if (is("WavelengthCentre")) {
        digHoloConfigSetWavelengthCentre(h, f0());
    } else if (is("WavelengthCount")) {
        run.wavelengthCount = i0();
    } else if (is("WavelengthStart")) {
        run.wavelengthStart = f0();
    } else if (is("WavelengthStop")) {
        run.wavelengthStop = f0();
    } else if (is("WavelengthOrdering")) {
        for (size_t a = 0; a < argc; a++) digHoloConfigSetWavelengthOrdering(h, (int)a, std::stoi(args[a]));
    } else if (is("MaxMG") || is("BasisGroupCount")) {
        digHoloConfigSetBasisGroupCount(h, i0());
    } else if (is("BasisType")) {
        digHoloConfigSetBasisType(h, i0());
    } else if (is("Waist") || is("BasisWaist")) {
        for (size_t a = 0; a < argc; a++) {
            const float v = std::stof(args[a]);
            run.waist = run.waist || v != 0;
            digHoloConfigSetBasisWaist(h, (int)a, v);
        }
        const int P = digHoloConfigGetPolCount(h);
        for (int p = (int)argc; p < P; p++) digHoloConfigSetBasisWaist(h, p, std::stof(args[argc - 1]));
    } else if (is("BatchAvgCount")) {
        digHoloConfigSetBatchAvgCount(h, i0());
    } else if (is("BatchAvgMode")) {
        digHoloConfigSetBatchAvgMode(h, i0());
    } else if (is("AutoAlignCentre")) {
        digHoloConfigSetAutoAlignBeamCentre(h, i0());
        run.autoAlign |= i0();
    } else if (is("AutoAlignDefocus")) {
        digHoloConfigSetAutoAlignDefocus(h, i0());
        run.autoAlign |= i0();
    } else if (is("AutoAlignTilt")) {
        digHoloConfigSetAutoAlignTilt(h, i0());
        run.autoAlign |= i0();
    } else if (is("AutoAlignWaist") || is("AutoAlignBasisWaist")) {
        digHoloConfigSetAutoAlignBasisWaist(h, i0());
        run.autoAlign |= i0();
    } else if (is("AutoAlignFourierWindowRadius")) {
        digHoloConfigSetAutoAlignFourierWindowRadius(h, i0());
        run.autoAlign |= i0();
    } else if (is("AutoAlignTol")) {
        digHoloConfigSetAutoAlignTol(h, f0());
    } else if (is("AutoAlignPolIndependence")) {
        digHoloConfigSetAutoAlignPolIndependence(h, i0());
    } else if (is("AutoAlignBasisMulConjTrans")) {
        digHoloConfigSetAutoAlignBasisMulConjTrans(h, i0());
    } else if (is("AutoAlignMode")) {
        digHoloConfigSetAutoAlignMode(h, i0());
    } else if (is("AutoAlignGoalIdx")) {
        digHoloConfigSetAutoAlignGoalIdx(h, i0());
    } else if (is("BasisCustomFilename")) {
        run.basisFile = args[0];
    } else if (is("BasisCustomModeCountIn")) {
        run.basisIn = i0();
    } else if (is("BasisCustomModeCountOut")) {
        run.basisOut = i0();
    } else if (is("RefCalibrationFilename")) {
        run.calibrationFile = args[0];
        run.calibration = true;
    } else if (is("BatchCalibrationFilename")) {
        run.batchCalibrationFile = args[0];
        run.batchCalibration = true;
    } else if (is("BatchCalibrationPolCount")) {
        run.batchCalPol = i0();
    } else if (is("BatchCalibrationBatchCount")) {
        run.batchCalCount = i0();
    } else if (is("FillFactorCorrection")) {
        digHoloConfigSetFillFactorCorrectionEnabled(h, i0());
    } else if (is("Viewport")) {
        run.viewport.clear();
        for (size_t a = 0; a < argc; a++) run.viewport.push_back(std::stoi(args[a]));
    }
    (void)errorCode;
    return true;
}

}  // namespace

extern "C" int digHoloRunBatchFromConfigFile(char* filename) {
    if (!filename) return ERR_NULLPOINTER;
    std::ifstream file(filename);
    const auto t0 = std::chrono::steady_clock::now();
    if (!file.is_open()) {
        fprintf(dh::console(), "File could not be opened. %s\n", filename);
        fflush(dh::console());
        return ERR_FILENOTFOUND;
    }
    // handle 0 when it exists, as the reference does (digHolo.cpp:16774-16782)
    const int h = (dhHandleCount() > 0 && digHoloConfigGetPolCount(0) > 0) ? 0 : digHoloCreate();
    Run run;
    int errorCode = 0;
    std::string line;
    while (std::getline(file, line) && !errorCode) {
        if (line.empty()) continue;
        if (line.back() == '\r') line.pop_back();
        std::istringstream in(line);
        std::string name, value;
        std::getline(in, name, '\t');
        std::vector<std::string> args;
        while (std::getline(in, value, '\t')) args.push_back(value);
        if (name == "FrameBufferFilename") {
            if (!args.empty()) {
                const int e = digHoloSetFrameBufferFromFile(h, args[0].c_str());
                if (e != ERR_SUCCESS) {
                    fprintf(dh::console(), "Fatal error. Aborting.\n");
                    fflush(dh::console());
                    return e;
                }
            } else {
                fprintf(dh::console(), "No file supplied. Generating test frames.\n");
                run.testFrames = 1;
            }
        }
        if (args.empty()) continue;
        try {
            applySetting(h, name, args, run, errorCode);
        } catch (const std::exception& ex) {
            fprintf(dh::console(), "%s\n", ex.what());
        }
    }
    file.close();
    int batchCount = digHoloConfigGetBatchCount(h);
    const int avgCount = digHoloConfigGetBatchAvgCount(h);
    int frameWidth = 0, frameHeight = 0;
    digHoloConfigGetFrameDimensions(h, &frameWidth, &frameHeight);
    if (!run.consoleFile.empty()) {
        std::vector<char> n(run.consoleFile.begin(), run.consoleFile.end());
        n.push_back(0);
        if (digHoloConsoleRedirectToFile(n.data()) != ERR_SUCCESS)
            fprintf(dh::console(), "Specified console output filename could not be created. %s\n", n.data());
    }
    if (run.wavelengthCount > 0)
        digHoloConfigSetWavelengthsLinearFrequency(h, run.wavelengthStart, run.wavelengthStop, run.wavelengthCount);
    if (run.calibration)
        digHoloConfigSetRefCalibrationFromFile(h, run.calibrationFile.c_str(), run.wavelengthCount, frameWidth, frameHeight);
    if (run.batchCalibration)
        digHoloConfigSetBatchCalibrationFromFile(h, run.batchCalibrationFile.c_str(), run.batchCalPol, run.batchCalCount);
    if (digHoloConfigGetBasisType(h) == 2) {
        std::ifstream bf(run.basisFile, std::ios::binary);
        if (bf && run.basisIn && run.basisOut) {
            bf.seekg(0, std::ios::end);
            const size_t bytes = (size_t)bf.tellg();
            bf.seekg(0, std::ios::beg);
            std::vector<float> t(bytes / 4);
            bf.read(reinterpret_cast<char*>(t.data()), (std::streamsize)(t.size() * 4));
            digHoloConfigSetBasisTypeCustom(h, run.basisIn, run.basisOut, reinterpret_cast<complex64*>(t.data()));
        } else {
            fprintf(dh::console(), "Error : BasisFilename could not be found. %s\n", run.basisFile.c_str());
        }
    }
    float* frameBuffer = nullptr;
    if (run.testFrames) {
        // simulated frames with the configured geometry (digHolo.cpp:17417-17556)
        int frames = batchCount, W = frameWidth, H = frameHeight, P = digHoloConfigGetPolCount(h);
        float ps = digHoloConfigGetFramePixelSize(h);
        std::vector<float> tX, tY, df, rcx, rcy, bcx, bcy, bw;
        float *ptX = nullptr, *ptY = nullptr, *pdf = nullptr, *prw = nullptr, *prcx = nullptr, *prcy = nullptr;
        float *pra = nullptr, *pbw = nullptr, *pbc = nullptr, *pbcx = nullptr, *pbcy = nullptr;
        if (run.tilt) {
            for (int p = 0; p < P; p++) { tX.push_back(digHoloConfigGetTilt(h, 0, p)); tY.push_back(digHoloConfigGetTilt(h, 1, p)); }
            ptX = tX.data();
            ptY = tY.data();
        }
        if (run.centre) {
            for (int p = 0; p < P; p++) {
                rcx.push_back(digHoloConfigGetBeamCentre(h, 0, p));
                rcy.push_back(digHoloConfigGetBeamCentre(h, 1, p));
            }
            bcx = rcx;
            bcy = rcy;
            prcx = rcx.data(); prcy = rcy.data(); pbcx = bcx.data(); pbcy = bcy.data();
        }
        if (run.defocus) {
            for (int p = 0; p < P; p++) df.push_back(digHoloConfigGetDefocus(h, p));
            pdf = df.data();
        }
        if (run.waist) {
            for (int p = 0; p < P; p++) bw.push_back(digHoloConfigGetBasisWaist(h, p));
            pbw = bw.data();
        }
        int G = digHoloConfigGetBasisGroupCount(h), levels = 16384, L = 1;
        float* wl = digHoloConfigGetWavelengths(h, &L);
        const int ordering = digHoloConfigGetWavelengthOrdering(h, 0);
        unsigned short* b16 = nullptr;
        frameBuffer = digHoloFrameSimulatorCreate(frames, &W, &H, &ps, &P, &ptX, &ptY, &pdf, &prw, &prcx, &prcy, &pra,
                                                  &G, &pbw, &pbc, &pbcx, &pbcy, &levels,
                                                  digHoloConfigGetFillFactorCorrectionEnabled(h), &wl, &L, ordering, 1,
                                                  &b16, "testFrame.bin");
    }
    digHoloSetBatchAvg(h, batchCount, frameBuffer, avgCount, digHoloConfigGetBatchAvgMode(h));
    int modeCount = 0, polCount = 0;
    float il = -1000, mdl = -1000, snr = -1000;
    double tAlign = 0, tBatch = 0;
    if (!run.autoAlign) {
        fprintf(dh::console(),
                "No AutoAlign parameters set(e.g. tilt, focus, waist, beam centre). Hence no AutoAlign will be performed. "
                "Using user specified digHolo parameters.\n");
        fflush(dh::console());
    } else {
        const auto a0 = std::chrono::steady_clock::now();
        digHoloAutoAlign(h);
        tAlign = std::chrono::duration<double>(std::chrono::steady_clock::now() - a0).count();
        il = digHoloAutoAlignGetMetric(h, METRIC_IL);
        mdl = digHoloAutoAlignGetMetric(h, METRIC_MDL);
        snr = digHoloAutoAlignGetMetric(h, METRIC_SNRAVG);
    }
    if (run.threadDiagnostic) digHoloConfigSetThreadCount(h, digHoloBenchmarkEstimateThreadCountOptimal(h, 15.0f));
    if (run.benchmark > 0) digHoloBenchmark(h, run.benchmark, nullptr);
    if (run.debug > 0) digHoloDebugRoutine(h);
    const int maxMG = digHoloConfigGetBasisGroupCount(h);
    if (!run.outCoefs.empty()) {
        const auto b0 = std::chrono::steady_clock::now();
        complex64* coefs = digHoloProcessBatch(h, &batchCount, &modeCount, &polCount);
        tBatch = std::chrono::duration<double>(std::chrono::steady_clock::now() - b0).count();
        if (coefs && batchCount && modeCount && polCount &&
            !writeBinary(run.outCoefs, coefs, sizeof(complex64), (size_t)batchCount * modeCount * polCount))
            fprintf(dh::console(), "Error : Could not open OutputFilenameCoefs %s\n", run.outCoefs.c_str());
    }
    int fieldW = 0, fieldH = 0;
    float *fx = nullptr, *fy = nullptr;
    if (!run.outBasis.empty() && maxMG) {
        complex64* bf = digHoloBasisGetFields(h, &modeCount, &polCount, &fx, &fy, &fieldW, &fieldH);
        if (bf && modeCount && polCount && fieldW && fieldH &&
            !writeBinary(run.outBasis, bf, sizeof(complex64), (size_t)modeCount * polCount * fieldW * fieldH))
            fprintf(dh::console(), "Error : Could not open OutputFilenameBasis %s\n", run.outBasis.c_str());
    }
    if (!run.outFields.empty()) {
        complex64* f = digHoloGetFields(h, &batchCount, &polCount, &fx, &fy, &fieldW, &fieldH);
        if (f && batchCount && polCount && fieldW && fieldH &&
            !writeBinary(run.outFields, f, sizeof(complex64), (size_t)batchCount * polCount * fieldW * fieldH))
            fprintf(dh::console(), "Error : Could not open OutputFilenameFields %s\n", run.outFields.c_str());
    }
    if (run.calibration && !run.outCalibration.empty()) {
        int cw = 0, ch = 0, cn = 0, cp = 0;
        float *cx = nullptr, *cy = nullptr;
        complex64* c = digHoloConfigGetRefCalibrationFields(h, &cn, &cp, &cx, &cy, &cw, &ch);
        writeBinary(run.outCalibration, c, sizeof(complex64), (size_t)cn * cp * cw * ch);
    }
    if (!run.viewport.empty() && !run.outViewport.empty()) {
        fprintf(dh::console(), "Viewport output %s not written: this library has no viewport renderer.\n",
                run.outViewport.c_str());
    }
    FILE* s = run.outSummary.empty() ? stdout : fopen(run.outSummary.c_str(), "w");
    if (s) {
        fprintf(s, "<SUMMARY>\n\r");
        for (int axis = 0; axis < 2; axis++) {
            fprintf(s, axis == 0 ? "BeamCentreX\t" : "BeamCentreY\t");
            for (int p = 0; p < polCount; p++)
                fprintf(s, p != polCount - 1 ? "%e\t" : "%e\n\r", digHoloConfigGetBeamCentre(h, axis, p));
        }
        for (int axis = 0; axis < 2; axis++) {
            fprintf(s, axis == 0 ? "TiltX\t" : "TiltY\t");
            for (int p = 0; p < polCount; p++)
                fprintf(s, p != polCount - 1 ? "%f\t" : "%f\n\r", digHoloConfigGetTilt(h, axis, p));
        }
        fprintf(s, "Defocus\t");
        for (int p = 0; p < polCount; p++) fprintf(s, p != polCount - 1 ? "%f\t" : "%f\n\r", digHoloConfigGetDefocus(h, p));
        fprintf(s, "Waist\t");
        for (int p = 0; p < polCount; p++) fprintf(s, p != polCount - 1 ? "%e\t" : "%e\n\r", digHoloConfigGetBasisWaist(h, p));
        fprintf(s, "FourierWindow\t%3.3f\n\r", digHoloConfigGetFourierWindowRadius(h));
        if (fieldW && fieldH) {
            fprintf(s, "FieldWidth\t%i\n\r", fieldW);
            fprintf(s, "FieldHeight\t%i\n\r", fieldH);
            if (!run.outX.empty()) writeBinary(run.outX, fx, sizeof(float), (size_t)fieldW);
            if (!run.outY.empty()) writeBinary(run.outY, fy, sizeof(float), (size_t)fieldH);
        }
        if (!run.autoAlign) {
            digHoloAutoAlignCalcMetrics(h);
            il = digHoloAutoAlignGetMetric(h, METRIC_IL);
            mdl = digHoloAutoAlignGetMetric(h, METRIC_MDL);
            snr = digHoloAutoAlignGetMetric(h, METRIC_SNRAVG);
        }
        fprintf(s, "IL\t%f\n\r", il);
        fprintf(s, "MDL\t%f\n\r", mdl);
        fprintf(s, "SNRAVG\t%f\n\r", snr);
        const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        fprintf(s, "Runtime (AutoAlign,sec. Hz)\t%f\t%f\n\r", tAlign, 1.0 / tAlign);
        fprintf(s, "Runtime (ProcessBatch,sec. Hz)\t%f\t%f\n\r", tBatch, 1.0 / tBatch);
        fprintf(s, "Runtime (Total,sec. Hz)\t%f\t%f\n\r", total, 1.0 / total);
        fprintf(s, "</SUMMARY>\n\r\n\r");
        fflush(s);
        if (s != stdout) fclose(s);
    } else {
        fprintf(dh::console(), "Error : Could not open OutputFilenameSummary %s\n\r", run.outSummary.c_str());
    }
    if (run.testFrames && frameBuffer) digHoloFrameSimulatorDestroy(frameBuffer);
    digHoloDestroy(h);
    return ERR_SUCCESS;
}
