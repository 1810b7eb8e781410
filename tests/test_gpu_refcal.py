"""Reference-wave calibration applied to the reconstructed fields
(digHoloConfigSetRefCalibrationIntensity / Field, digHolo.h:369-437;
applied at digHolo.cpp:8736-8758 with the planes of digHolo.cpp:6729-6830,
8253-8285).

Against the oracle (ref_cal_planes and process_batch with the stored
factors, pinned to the reference build in test_oracle_pin) and, where the
reference build exists, against the reference itself on the same frames
(in a child process: the reference's calibrated batches can corrupt its
heap, helpers.reference_calibrated):

* the calibration planes digHoloConfigGetRefCalibrationFields returns:
  relative L2 <= 1e-5 against the oracle and the reference;
* the calibrated batch: int16 fields within 2 LSB, fields relative L2 <= 5e-5,
  coefficients relative L2 <= 5e-5 (the reference's unscaled 16-row
  coefficients, digHolo.cpp:2318-2331, taken into account);
* full-resolution fields beyond one thread block (band kernel) as well;
* disabling the calibration gives the plain batch back; device frames give
  the host-frame result; a multi-wavelength batch with one calibration item
  matches the reference's.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
import ref_lib
from digholo_b200 import api
from helpers import (config_for, make_case, ref_calibration, ref_calibration_planes, reference_calibrated, rel_l2,
                     set_ref_calibration)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _run(L, cfg, frames, kind, cal, keep=False):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    set_ref_calibration(L, h, cfg, kind, cal)
    # the library keeps only the pointer: the array must outlive the processing
    frames = np.ascontiguousarray(frames if frames.dtype == np.uint16 else frames.astype(np.float32))
    assert api.set_batch(L, h, frames) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    assert cp, (L.digHoloB200GetLastError(h) if hasattr(L, "digHoloB200GetLastError") else "reference: no coefficients")
    out = api.read_outputs(L, h, frames.shape[0], cp, m.value, p.value, True)
    out["planes"] = ref_calibration_planes(L, h)
    out["h"] = h
    if not keep:
        L.digHoloDestroy(h)
    return out


def _compare(g, ref, cfg, tol=5e-5):
    dmax = max(np.abs(g["R"].astype(int) - ref["R"]).max(), np.abs(g["I"].astype(int) - ref["I"]).max())
    assert dmax <= 2
    assert rel_l2(g["field"], ref["field"]) <= tol
    return dmax


CASES = [("plain_320x256_f32_1pol", 1, "intensity", 1), ("plain_320x256_f32_1pol", 0, "field", 2),
         ("batched_640x512_u16_2pol", 1, "field", 1), ("batched_640x512_u16_2pol", 0, "intensity", 3)]


@pytest.mark.parametrize("workload,mode,kind,count", CASES, ids=[str(i) for i in range(len(CASES))])
def test_calibrated_batch_matches_oracle_and_reference(lib, workload, mode, kind, count):
    hol = make_case(workload, 6)
    cfg = config_for(hol, mode)
    cal = ref_calibration(cfg, kind, count)
    g = _run(lib, cfg, hol.frames, kind, cal)
    op = O.ref_cal_planes(cfg)
    assert g["planes"] is not None and g["planes"].shape == op.shape
    ep = rel_l2(g["planes"], op)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    dmax = max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max())
    ef = rel_l2(g["field"], o["field"])
    ec = rel_l2(g["coefs"], o["coefs"])
    print("%s mode %d %s x%d: planes %.2e, int16 max diff %d, fields %.2e, coefs %.2e"
          % (workload, mode, kind, count, ep, dmax, ef, ec))
    assert ep <= 1e-5
    assert dmax <= 2 and ef <= 5e-5 and ec <= 5e-5
    # the calibration is visible in the coefficients
    plain = O.process_batch(hol.frames, config_for(hol, mode), quantised=True)
    assert rel_l2(plain["coefs"], g["coefs"]) > 3e-3
    if ref_lib.available():
        r = reference_calibrated(workload, 6, mode, kind, count)
        assert rel_l2(g["planes"], r["planes"]) <= 1e-5
        _compare(g, r, cfg)
        gc = g["coefs"]
        if mode == 1 and g["R"].shape[-2] == 16:
            gc = O.reference_unscaled_16(gc.astype(np.complex128), cfg, {"x": g["x"], "y": g["y"], "scale": g["scale"].T})
        assert rel_l2(gc, r["coefs"]) <= 5e-5


def test_disable_restores_plain_batch(lib):
    hol = make_case("batched_640x512_u16_2pol", 4)
    cfg = config_for(hol, 1)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    plain = api.run_batch(lib, h, hol.frames)["coefs"]
    set_ref_calibration(lib, h, cfg, "intensity", ref_calibration(cfg, "intensity"))
    assert lib.digHoloConfigGetRefCalibrationEnabled(h) == 1
    cal = api.run_batch(lib, h, hol.frames)["coefs"]
    assert rel_l2(cal, plain) > 1e-3
    assert lib.digHoloConfigSetRefCalibrationEnabled(h, 0) == 0
    again = api.run_batch(lib, h, hol.frames)["coefs"]
    assert np.array_equal(again, plain)
    # a calibration of another frame size does not apply (digHolo.cpp:8242)
    other = ref_calibration(config_for(make_case("plain_320x256_f32_1pol", 1), 1), "intensity")
    assert lib.digHoloConfigSetRefCalibrationIntensity(h, other.ctypes.data_as(C.POINTER(C.c_ushort)), 1,
                                                       other.shape[2], other.shape[1]) == 0
    assert np.array_equal(api.run_batch(lib, h, hol.frames)["coefs"], plain)


def test_device_frames_match_host_frames(lib):
    """Device-resident frames (direct launches, then graph replay) give the
    host-frame batch's coefficients exactly."""
    import torch
    hol = make_case("batched_640x512_u16_2pol", 8)
    cfg = config_for(hol, 1)
    cal = ref_calibration(cfg, "field", 1)
    host = _run(lib, cfg, hol.frames, "field", cal)["coefs"]
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    set_ref_calibration(lib, h, cfg, "field", cal)
    t = torch.from_numpy(np.ascontiguousarray(hol.frames.astype(np.uint16)).view(np.int16)).cuda()
    B = hol.frames.shape[0]
    for _ in range(3):   # direct launches, capture, replay
        lib.digHoloSetBatchUint16(h, B, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_ushort)), 0)
        b, m, p = C.c_int(), C.c_int(), C.c_int()
        cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
        assert cp, lib.digHoloB200GetLastError(h)
        got = np.ctypeslib.as_array(cp, shape=(b.value * m.value * p.value * 2,)).copy().view(np.complex64)
        assert np.array_equal(got.reshape(host.shape), host)


@pytest.mark.parametrize("workload,frames,window", [("batched_640x512_u16_2pol", 3, (256, 256)),
                                                    ("largefield_2048_u16_2pol", 1, None)])
def test_large_full_resolution_fields(lib, workload, frames, window):
    """Full-resolution fields beyond one thread block (256 x 256, and the
    512 x 512 fields of 2048 x 2048 frames): the calibration is applied by the
    64-row band kernel k_field_big; the same bounds against the oracle (and,
    for the 256 x 256 fields, the reference; the oracle is pinned to the
    reference on the 512 x 512 case in test_oracle_pin)."""
    hol = make_case(workload, frames)
    cfg = config_for(hol, 0)
    if window:
        cfg.fft_window = window
    cal = ref_calibration(cfg, "intensity", 1)
    g = _run(lib, cfg, hol.frames, "intensity", cal)
    op = O.ref_cal_planes(cfg)
    assert rel_l2(g["planes"], op) <= 1e-5
    o = O.process_batch(hol.frames, cfg, quantised=True)
    dmax = max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max())
    ef, ec = rel_l2(g["field"], o["field"]), rel_l2(g["coefs"], o["coefs"])
    print("%s full resolution %s: int16 max diff %d, fields %.2e, coefs %.2e" % (workload, g["R"].shape, dmax, ef, ec))
    assert dmax <= 2 and ef <= 5e-5 and ec <= 5e-5
    if ref_lib.available() and window:
        r = reference_calibrated(workload, frames, 0, "intensity", 1, window[0])
        assert rel_l2(g["planes"], r["planes"]) <= 1e-5
        _compare(g, r, cfg)
        assert rel_l2(g["coefs"], r["coefs"]) <= 5e-5


def test_sweep_with_one_item_matches_reference(lib):
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    hol = make_case("batched_640x512_u16_2pol", 6)
    cfg = config_for(hol, 1)
    cal = ref_calibration(cfg, "intensity", 1)
    lams = [1550e-9, 1575e-9, 1600e-9]
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    set_ref_calibration(lib, h, cfg, "intensity", cal)
    assert api.set_batch(lib, h, hol.frames) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    arr = (C.c_float * 3)(*lams)
    cp = lib.digHoloProcessBatchWavelengthSweepArbitrary(h, C.byref(b), C.byref(m), C.byref(p), arr, 3)
    assert cp, lib.digHoloB200GetLastError(h)
    g = api.read_outputs(lib, h, 6, cp, m.value, p.value, True)
    lib.digHoloDestroy(h)
    r = reference_calibrated("batched_640x512_u16_2pol", 6, 1, "intensity", 1, sweep=lams)
    _compare(g, r, cfg)
    gc = O.reference_unscaled_16(g["coefs"].astype(np.complex128), cfg, {"x": g["x"], "y": g["y"], "scale": g["scale"].T})
    assert rel_l2(gc, r["coefs"]) <= 5e-5
