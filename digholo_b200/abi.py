"""C-ABI prototype table and ctypes binder for the digHolo interface.

The table lists every entry point declared by the reference's public header
(digHolo.h:209-2084, the ``EXT_C`` declarations) with its return and argument
types, spelled as in that header.  The same table binds two libraries that
share the interface:

* this project's ``libdigholo_b200.so`` (plain ``extern "C"`` names), and
* the reference build used only by the tests (C++-mangled names, because
  ``EXT_C`` expands to nothing on Linux, digHolo.h:148-156), through a
  ``resolver`` that maps plain names to mangled ones.

``complex64`` is ``float[2]`` (digHolo.h:163), so ``complex64*`` is bound as a
plain ``float*`` and arrays are read with stride 2.
"""
import ctypes as C

PROTOTYPES = {
    "digHoloCreate": ("int", ()),
    "digHoloDestroy": ("int", ('int',)),
    "digHoloSetFrameBuffer": ("int", ('int', 'float*')),
    "digHoloGetFrameBuffer": ("float*", ('int',)),
    "digHoloSetFrameBufferUint16": ("int", ('int', 'unsigned short*', 'int')),
    "digHoloGetFrameBufferUint16": ("unsigned short*", ('int', 'int*')),
    "digHoloSetFrameBufferFromFile": ("int", ('int', 'const char*')),
    "digHoloConfigSetFrameDimensions": ("int", ('int', 'int', 'int')),
    "digHoloConfigGetFrameDimensions": ("int", ('int', 'int*', 'int*')),
    "digHoloConfigSetFramePixelSize": ("int", ('int', 'float')),
    "digHoloConfigGetFramePixelSize": ("float", ('int',)),
    "digHoloConfigSetPolCount": ("int", ('int', 'int')),
    "digHoloConfigGetPolCount": ("int", ('int',)),
    "digHoloConfigSetRefCalibrationIntensity": ("int", ('int', 'unsigned short*', 'int', 'int', 'int')),
    "digHoloConfigSetRefCalibrationField": ("int", ('int', 'complex64*', 'int', 'int', 'int')),
    "digHoloConfigSetRefCalibrationFromFile": ("int", ('int', 'const char*', 'int', 'int', 'int')),
    "digHoloConfigSetRefCalibrationEnabled": ("int", ('int', 'int')),
    "digHoloConfigGetRefCalibrationEnabled": ("int", ('int',)),
    "digHoloConfigGetRefCalibrationFields": ("complex64*", ('int', 'int*', 'int*', 'float**', 'float**', 'int*', 'int*')),
    "digHoloConfigSetFillFactorCorrectionEnabled": ("int", ('int', 'int')),
    "digHoloConfigGetFillFactorCorrectionEnabled": ("int", ('int',)),
    "digHoloSetBatch": ("int", ('int', 'int', 'float*')),
    "digHoloSetBatchAvg": ("int", ('int', 'int', 'float*', 'int', 'int')),
    "digHoloSetBatchUint16": ("int", ('int', 'int', 'unsigned short*', 'int')),
    "digHoloSetBatchAvgUint16": ("int", ('int', 'int', 'unsigned short*', 'int', 'int', 'int')),
    "digHoloConfigSetBatchCount": ("int", ('int', 'int')),
    "digHoloConfigGetBatchCount": ("int", ('int',)),
    "digHoloConfigSetBatchAvgCount": ("int", ('int', 'int')),
    "digHoloConfigGetBatchAvgCount": ("int", ('int',)),
    "digHoloConfigSetBatchCalibration": ("int", ('int', 'complex64*', 'int', 'int')),
    "digHoloConfigGetBatchCalibration": ("complex64*", ('int', 'int*', 'int*')),
    "digHoloConfigSetBatchCalibrationFromFile": ("int", ('int', 'const char*', 'int', 'int')),
    "digHoloConfigSetBatchCalibrationEnabled": ("int", ('int', 'int')),
    "digHoloConfigGetBatchCalibrationEnabled": ("int", ('int',)),
    "digHoloConfigSetBatchAvgMode": ("int", ('int', 'int')),
    "digHoloConfigGetBatchAvgMode": ("int", ('int',)),
    "digHoloConfigSetfftWindowSize": ("int", ('int', 'int', 'int')),
    "digHoloConfigGetfftWindowSize": ("int", ('int', 'int*', 'int*')),
    "digHoloConfigSetfftWindowSizeX": ("int", ('int', 'int')),
    "digHoloConfigGetfftWindowSizeX": ("int", ('int',)),
    "digHoloConfigGetfftWindowSizeY": ("int", ('int',)),
    "digHoloConfigSetfftWindowSizeY": ("int", ('int', 'int')),
    "digHoloConfigSetFourierWindowRadius": ("int", ('int', 'float')),
    "digHoloConfigGetFourierWindowRadius": ("float", ('int',)),
    "digHoloConfigSetIFFTResolutionMode": ("int", ('int', 'int')),
    "digHoloConfigGetIFFTResolutionMode": ("int", ('int',)),
    "digHoloConfigSetWavelengthCentre": ("int", ('int', 'float')),
    "digHoloConfigGetWavelengthCentre": ("float", ('int',)),
    "digHoloConfigSetWavelengths": ("int", ('int', 'float*', 'int')),
    "digHoloConfigSetWavelengthsLinearFrequency": ("int", ('int', 'float', 'float', 'int')),
    "digHoloConfigGetWavelengths": ("float*", ('int', 'int*')),
    "digHoloConfigSetWavelengthOrdering": ("int", ('int', 'int', 'int')),
    "digHoloConfigGetWavelengthOrdering": ("int", ('int', 'int')),
    "digHoloConfigSetAutoAlignBeamCentre": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignBeamCentre": ("int", ('int',)),
    "digHoloConfigSetAutoAlignDefocus": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignDefocus": ("int", ('int',)),
    "digHoloConfigSetAutoAlignTilt": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignTilt": ("int", ('int',)),
    "digHoloConfigSetAutoAlignBasisWaist": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignBasisWaist": ("int", ('int',)),
    "digHoloConfigSetAutoAlignFourierWindowRadius": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignFourierWindowRadius": ("int", ('int',)),
    "digHoloConfigSetAutoAlignTol": ("int", ('int', 'float')),
    "digHoloConfigGetAutoAlignTol": ("float", ('int',)),
    "digHoloConfigSetAutoAlignPolIndependence": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignPolIndependence": ("int", ('int',)),
    "digHoloConfigSetAutoAlignBasisMulConjTrans": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignBasisMulConjTrans": ("int", ('int',)),
    "digHoloConfigSetAutoAlignMode": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignMode": ("int", ('int',)),
    "digHoloConfigSetAutoAlignGoalIdx": ("int", ('int', 'int')),
    "digHoloConfigGetAutoAlignGoalIdx": ("int", ('int',)),
    "digHoloAutoAlign": ("float", ('int',)),
    "digHoloAutoAlignGetMetric": ("float", ('int', 'int')),
    "digHoloAutoAlignGetMetrics": ("float*", ('int', 'int')),
    "digHoloAutoAlignCalcMetrics": ("int", ('int',)),
    "digHoloConfigSetBeamCentre": ("int", ('int', 'int', 'int', 'float')),
    "digHoloConfigGetBeamCentre": ("float", ('int', 'int', 'int')),
    "digHoloConfigSetTilt": ("int", ('int', 'int', 'int', 'float')),
    "digHoloConfigGetTilt": ("float", ('int', 'int', 'int')),
    "digHoloConfigSetDefocus": ("int", ('int', 'int', 'float')),
    "digHoloConfigGetDefocus": ("float", ('int', 'int')),
    "digHoloConfigSetPolLockTilt": ("int", ('int', 'int')),
    "digHoloConfigGetPolLockTilt": ("int", ('int',)),
    "digHoloConfigSetPolLockDefocus": ("int", ('int', 'int')),
    "digHoloConfigGetPolLockDefocus": ("int", ('int',)),
    "digHoloConfigSetPolLockBasisWaist": ("int", ('int', 'int')),
    "digHoloConfigGetPolLockBasisWaist": ("int", ('int',)),
    "digHoloConfigSetBasisGroupCount": ("int", ('int', 'int')),
    "digHoloConfigGetBasisGroupCount": ("int", ('int',)),
    "digHoloConfigSetBasisWaist": ("int", ('int', 'int', 'float')),
    "digHoloConfigGetBasisWaist": ("float", ('int', 'int')),
    "digHoloConfigSetBasisTypeHG": ("int", ('int',)),
    "digHoloConfigSetBasisTypeLG": ("int", ('int',)),
    "digHoloConfigSetBasisTypeCustom": ("int", ('int', 'int', 'int', 'complex64*')),
    "digHoloConfigSetBasisType": ("int", ('int', 'int')),
    "digHoloConfigGetBasisType": ("int", ('int',)),
    "digHoloProcessBatch": ("complex64*", ('int', 'int*', 'int*', 'int*')),
    "digHoloProcessBatchFrequencySweepLinear": ("complex64*", ('int', 'int*', 'int*', 'int*', 'float', 'float', 'int')),
    "digHoloProcessBatchWavelengthSweepArbitrary": ("complex64*", ('int', 'int*', 'int*', 'int*', 'float*', 'int')),
    "digHoloGetFields": ("complex64*", ('int', 'int*', 'int*', 'float**', 'float**', 'int*', 'int*')),
    "digHoloGetFields16": ("int", ('int', 'int*', 'int*', 'short**', 'short**', 'float**', 'float**', 'float**', 'int*', 'int*')),
    "digHoloBasisGetFields": ("complex64*", ('int', 'int*', 'int*', 'float**', 'float**', 'int*', 'int*')),
    "digHoloBasisGetCoefs": ("complex64*", ('int', 'int*', 'int*', 'int*')),
    "digHoloBatchGetSummary": ("int", ('int', 'int', 'int*', 'int*', 'int*', 'float**', 'int*', 'int*', 'float**', 'float**', 'float**')),
    "digHoloProcessFFT": ("int", ('int',)),
    "digHoloProcessIFFT": ("int", ('int',)),
    "digHoloProcessRemoveTilt": ("int", ('int',)),
    "digHoloProcessBasisExtractCoefs": ("int", ('int',)),
    "digHoloGetFourierPlaneFull": ("complex64*", ('int', 'int*', 'int*', 'int*', 'int*')),
    "digHoloGetFourierPlaneWindow": ("complex64*", ('int', 'int*', 'int*', 'int*', 'int*')),
    "digHoloConfigSetThreadCount": ("int", ('int', 'int')),
    "digHoloConfigGetThreadCount": ("int", ('int',)),
    "digHoloBenchmarkEstimateThreadCountOptimal": ("int", ('int', 'float')),
    "digHoloBenchmark": ("float", ('int', 'float', 'float*')),
    "digHoloConfigSetFFTWPlanMode": ("int", ('int', 'int')),
    "digHoloConfigGetFFTWPlanMode": ("int", ('int',)),
    "digHoloFFTWWisdomForget": ("int", ()),
    "digHoloFFTWWisdomFilename": ("int", ('const char*',)),
    "digHoloGetViewport": ("unsigned char*", ('int', 'int', 'int', 'int*', 'int*', 'char**')),
    "digHoloGetViewportToFile": ("int", ('int', 'int', 'int', 'int*', 'int*', 'char**', 'const char*')),
    "digHoloConfigSetVerbosity": ("int", ('int', 'int')),
    "digHoloConfigGetVerbosity": ("int", ('int',)),
    "digHoloConsoleRedirectToFile": ("int", ('char*',)),
    "digHoloConsoleRestore": ("int", ()),
    "digHoloRunBatchFromConfigFile": ("int", ('char*',)),
    "digHoloConfigBackupSave": ("int", ('int',)),
    "digHoloConfigBackupLoad": ("int", ('int',)),
    "digHoloDebugRoutine": ("void", ('int',)),
    "digHoloFrameSimulatorCreate": ("float*", ('int', 'int*', 'int*', 'float*', 'int*', 'float**', 'float**', 'float**', 'float**', 'float**', 'float**', 'complex64**', 'int*', 'float**', 'complex64**', 'float**', 'float**', 'int*', 'int', 'float**', 'int*', 'int', 'int', 'unsigned short**', 'const char*')),
    "digHoloFrameSimulatorCreateSimple": ("float*", ('int', 'int', 'int', 'float', 'int', 'float', 'int')),
    "digHoloFrameSimulatorDestroy": ("int", ('float*',)),
    "digHoloConfigGetZernCoefs": ("float**", ('int',)),
    "digHoloConfigGetZernCount": ("int", ('int',)),
}

_CTYPES = {
    "void": None,
    "int": C.c_int,
    "float": C.c_float,
    "int*": C.POINTER(C.c_int),
    "float*": C.POINTER(C.c_float),
    "float**": C.POINTER(C.POINTER(C.c_float)),
    "complex64*": C.POINTER(C.c_float),
    "complex64**": C.POINTER(C.POINTER(C.c_float)),
    "short**": C.POINTER(C.POINTER(C.c_short)),
    "unsigned short*": C.POINTER(C.c_ushort),
    "unsigned short**": C.POINTER(C.POINTER(C.c_ushort)),
    "unsigned char*": C.POINTER(C.c_ubyte),
    "char*": C.c_char_p,
    "const char*": C.c_char_p,
    "char**": C.POINTER(C.c_char_p),
}


def ctype_of(spelling):
    """ctypes type for a C type spelled as in the reference header."""
    return _CTYPES[spelling]


class Bound:
    """Namespace of bound entry points; ``missing`` lists table names the library lacks."""

    def __init__(self):
        self.missing = []


def bind(lib, resolver=None, names=None):
    """Bind the entry points of ``lib`` (a ``ctypes.CDLL``) listed in PROTOTYPES.

    ``resolver(name)`` returns the exported symbol for a plain name, or None;
    by default the plain name itself is looked up.  Entry points the library
    does not export are recorded in ``Bound.missing`` instead of raising.
    """
    out = Bound()
    for name, (ret, args) in PROTOTYPES.items():
        if names is not None and name not in names:
            continue
        sym = resolver(name) if resolver else name
        fn = None
        if sym is not None:
            try:
                fn = getattr(lib, sym)
            except AttributeError:
                fn = None
        if fn is None:
            out.missing.append(name)
            continue
        fn.restype = ctype_of(ret)
        fn.argtypes = [ctype_of(a) for a in args]
        setattr(out, name, fn)
    return out
