"""The C ABI without a GPU: the library loads, exports every entry point
include/digHolo.h declares, and its configuration setters/getters behave like
the reference's (same return codes, clamping and stored values)."""
import ctypes as C
import os
import re

import pytest

import ref_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "digHolo.h")).read()
    return sorted(set(re.findall(r"\b(digHolo\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def test_library_exports_every_declared_symbol():
    import digholo_b200
    raw = C.CDLL(digholo_b200.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(raw, n)]
    assert not missing, missing
    assert len(_declared()) >= 100


def test_prototype_table_covers_reference_entry_points(lib):
    from digholo_b200 import abi
    declared = set(_declared())
    ref_names = [n for n in declared if not n.startswith("digHoloB200")]
    assert all(n in abi.PROTOTYPES for n in ref_names)


# (call, args) sequences whose return values must equal the reference's
SEQUENCE = [
    ("digHoloConfigSetFrameDimensions", (640, 512)),
    ("digHoloConfigSetFrameDimensions", (641, 512)),
    ("digHoloConfigSetFramePixelSize", (20e-6,)),
    ("digHoloConfigSetFramePixelSize", (-1.0,)),
    ("digHoloConfigSetPolCount", (2,)),
    ("digHoloConfigSetPolCount", (3,)),
    ("digHoloConfigGetPolCount", ()),
    ("digHoloConfigSetfftWindowSizeX", (130,)),
    ("digHoloConfigSetfftWindowSizeY", (-4,)),
    ("digHoloConfigGetfftWindowSizeX", ()),
    ("digHoloConfigSetfftWindowSize", (100, 70)),
    ("digHoloConfigGetfftWindowSizeY", ()),
    ("digHoloConfigSetFourierWindowRadius", (0.0,)),
    ("digHoloConfigSetFourierWindowRadius", (0.3,)),
    ("digHoloConfigSetIFFTResolutionMode", (2,)),
    ("digHoloConfigSetIFFTResolutionMode", (1,)),
    ("digHoloConfigGetIFFTResolutionMode", ()),
    ("digHoloConfigSetWavelengthCentre", (1550e-9,)),
    ("digHoloConfigSetWavelengthCentre", (0.0,)),
    ("digHoloConfigSetBeamCentre", (0, 1, 1e-4)),
    ("digHoloConfigSetBeamCentre", (2, 0, 1e-4)),
    ("digHoloConfigSetBeamCentre", (0, 5, 1e-4)),
    ("digHoloConfigGetBeamCentre", (0, 1)),
    ("digHoloConfigSetTilt", (1, 0, 0.5)),
    ("digHoloConfigSetTilt", (3, 0, 0.5)),
    ("digHoloConfigGetTilt", (1, 0)),
    ("digHoloConfigSetDefocus", (1, 0.25)),
    ("digHoloConfigSetDefocus", (4, 0.25)),
    ("digHoloConfigGetDefocus", (1,)),
    ("digHoloConfigSetBasisGroupCount", (-7,)),
    ("digHoloConfigGetBasisGroupCount", ()),
    ("digHoloConfigSetBasisWaist", (1, 300e-6)),
    ("digHoloConfigGetBasisWaist", (0,)),
    ("digHoloConfigSetBasisWaist", (0, -1.0)),
    ("digHoloConfigSetPolLockTilt", (5,)),
    ("digHoloConfigGetPolLockTilt", ()),
    ("digHoloConfigSetBatchCount", (0,)),
    ("digHoloConfigGetBatchCount", ()),
    ("digHoloConfigSetBatchAvgMode", (7,)),
    ("digHoloConfigGetBatchAvgMode", ()),
    ("digHoloConfigSetFillFactorCorrectionEnabled", (0,)),
    ("digHoloConfigGetFillFactorCorrectionEnabled", ()),
    ("digHoloConfigSetAutoAlignMode", (5,)),
    ("digHoloConfigSetAutoAlignGoalIdx", (1,)),
    ("digHoloConfigGetAutoAlignGoalIdx", ()),
    ("digHoloConfigSetWavelengthsLinearFrequency", (1500e-9, 1600e-9, 0)),
    ("digHoloConfigSetWavelengthsLinearFrequency", (1500e-9, 1600e-9, -3)),
    ("digHoloConfigSetWavelengthsLinearFrequency", (1500e-9, 1600e-9, 5)),
    ("digHoloConfigSetWavelengthOrdering", (0, 1)),
    ("digHoloConfigSetWavelengthOrdering", (2, 1)),
    ("digHoloConfigSetWavelengthOrdering", (1, 3)),
    ("digHoloConfigGetWavelengthOrdering", (0,)),
    ("digHoloConfigGetWavelengthOrdering", (1,)),
    ("digHoloConfigGetWavelengthOrdering", (7,)),
    ("digHoloConfigBackupSave", ()),
    ("digHoloConfigBackupLoad", ()),
    ("digHoloConfigGetZernCount", ()),
    ("digHoloConfigSetRefCalibrationIntensity", (None, 1, 16, 16)),
    ("digHoloConfigGetRefCalibrationEnabled", ()),
    ("digHoloConfigSetRefCalibrationEnabled", (1,)),
    ("digHoloConfigGetRefCalibrationEnabled", ()),
    ("digHoloConfigSetRefCalibrationFromFile", (b"no_such_calibration.bin", 1, 16, 16)),
    ("digHoloConfigGetRefCalibrationEnabled", ()),
    ("digHoloConfigSetBatchCalibrationFromFile", (b"no_such_calibration.bin", 1, 4)),
    ("digHoloSetFrameBufferFromFile", (b"no_such_frames.bin",)),
]


def _run_sequence(L):
    h = L.digHoloCreate()
    out = []
    for name, args in SEQUENCE:
        v = getattr(L, name)(h, *args)
        out.append(round(v, 12) if isinstance(v, float) else v)
    return out


def test_config_semantics_match_reference(lib):
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    ours = _run_sequence(lib)
    ref = _run_sequence(ref_lib.load())
    diffs = [(SEQUENCE[i][0], SEQUENCE[i][1], a, b) for i, (a, b) in enumerate(zip(ours, ref)) if a != b]
    assert not diffs, diffs


def test_wavelengths_before_processing(lib):
    """Before any processing there is no wavelength array in use: NULL and a
    zero count, as in the reference (digHolo.cpp:5056-5068); the setters'
    return codes are compared in the sequence above."""
    out = []
    libs = [lib] + ([ref_lib.load()] if ref_lib.available() else [])
    for L in libs:
        h = L.digHoloCreate()
        assert L.digHoloConfigSetWavelengthsLinearFrequency(h, 1500e-9, 1600e-9, 7) == 0
        n = C.c_int(5)
        p = L.digHoloConfigGetWavelengths(h, C.byref(n))
        out.append((bool(p), n.value))
        if L is lib:
            L.digHoloDestroy(h)   # the reference's Destroy faults after this sequence; its handle is left
    assert all(v == (False, 0) for v in out)


def test_invalid_handle_returns(lib):
    b, m, p = C.c_int(9), C.c_int(9), C.c_int(9)
    assert not lib.digHoloProcessBatch(12345, C.byref(b), C.byref(m), C.byref(p))
    assert (b.value, m.value, p.value) == (0, 0, 0)
    assert lib.digHoloConfigSetPolCount(-1, 1) == 2
    assert lib.digHoloConfigGetPolCount(-1) == 0
    assert lib.digHoloConfigGetFramePixelSize(999) == 0.0


def test_processing_without_frames_fails(lib):
    h = lib.digHoloCreate()
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    assert not lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    assert lib.digHoloSetBatch(h, 4, None) == 3


def test_no_cpu_fallback(lib):
    """On a machine without a CUDA device the batch path reports an error instead of computing."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    import numpy as np
    h = lib.digHoloCreate()
    frames = np.zeros((2, 256, 320), dtype=np.float32)
    lib.digHoloSetBatch(h, 2, frames.ctypes.data_as(C.POINTER(C.c_float)))
    lib.digHoloConfigSetBasisGroupCount(h, 3)
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    assert not lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    assert b"CUDA" in lib.digHoloB200GetLastError(h)


def _mangled_aliases():
    path = os.path.join(ROOT, "digholo_b200", "csrc", "_build", "mangled.ld")
    out = {}
    for line in open(path):
        m = re.match(r"(\S+) = (\w+);", line.strip())
        if m:
            out[m.group(2)] = m.group(1)
    return out


def test_cxx_mangled_aliases_exported():
    """Every reference entry point is exported under its C++-mangled name
    too (the reference's Linux exports are mangled: EXT_C is empty there,
    digHolo.h:148-156), as an alias of the C-linkage function."""
    import digholo_b200
    raw = C.CDLL(digholo_b200.LIB_PATH)
    aliases = _mangled_aliases()
    ref_names = [n for n in _declared() if not n.startswith("digHoloB200")]
    assert sorted(aliases) == sorted(ref_names)
    missing = [m for m in aliases.values() if not hasattr(raw, m)]
    assert not missing, missing


def test_cxx_mangled_names_match_reference_build():
    """The mangled names equal the reference build's own exports for every
    entry point both libraries have, and calls through them behave like the
    C names (a g++-built caller of the reference relinks unchanged)."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    import digholo_b200
    from digholo_b200 import abi
    table = ref_lib._symbol_map()
    aliases = _mangled_aliases()
    shared = [n for n in table if n in aliases]
    assert len(shared) >= 100
    assert {n: table[n] for n in shared} == {n: aliases[n] for n in shared}
    raw = C.CDLL(digholo_b200.LIB_PATH)
    M = abi.bind(raw, resolver=table.get)
    h = M.digHoloCreate()
    assert h >= 0
    assert M.digHoloConfigSetFrameDimensions(h, 640, 512) == 0
    w, hh = C.c_int(), C.c_int()
    assert M.digHoloConfigGetFrameDimensions(h, C.byref(w), C.byref(hh)) == 0
    assert (w.value, hh.value) == (640, 512)
    assert M.digHoloConfigSetPolCount(h, 2) == 0 and M.digHoloConfigGetPolCount(h) == 2
    assert M.digHoloDestroy(h) == 0
