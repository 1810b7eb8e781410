"""Full-resolution fields by bands of 64 rows (inverse kernel 4): a
statistics pass, a quantising pass with the overlap (split-BF16 tensor cores
or FP32 CUDA cores) and a coefficient sum.  Fields larger than 128 x 128 take
this path by default; digHoloB200SetInverseKernel(h, 2) forces it for smaller
fields.

Cases: 512 x 512 uint16 frames with a 256 x 256 FFT window (32 x 32 IFFT
window); 640 x 512 float frames, two polarisations, a 256 x 128 window
(32 x 16 IFFT window, rectangular); the 640 x 512 uint16 two-polarisation
batch with its 128 x 128 window forced onto the bands.  Tolerances as in
test_gpu_parity: int16 fields within 2 LSB of the quantised oracle, field
relative L2 <= 5e-5, scales relative <= 1e-5, coefficients relative L2 <=
5e-5 (FP32) or 1e-4 (split-BF16), FP32 fields before rounding relative L2 <=
1e-5 against the unquantised oracle.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
from digholo_b200 import api, synth
from helpers import config_for, make_case, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _case(name):
    if name == "square256":
        return synth.generate(frame_count=6, frame_width=512, frame_height=512, pol_count=1, max_mg=9, waist=250e-6,
                              snr_db=30, window=(256, 256), dtype="uint16", seed=11)
    if name == "rect256x128":
        return synth.generate(frame_count=6, frame_width=640, frame_height=512, pol_count=2, max_mg=12, waist=220e-6,
                              snr_db=30, window=(256, 128), dtype="float32", seed=12)
    return make_case("batched_640x512_u16_2pol", 6)


def _run(L, hol, cfg, inverse, overlap):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    assert L.digHoloB200SetInverseKernel(h, inverse) == 0
    assert L.digHoloB200SetOverlapKernel(h, overlap) == 0
    L.digHoloB200SetKeepField32(h, 1)
    out = api.run_batch(L, h, hol.frames)
    assert out["coefs"] is not None, L.digHoloB200GetLastError(h)
    out["kernel"] = L.digHoloB200GetInverseKernel(h)
    out["overlap"] = L.digHoloB200GetOverlapKernel(h)
    b, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    fp = L.digHoloB200GetFields32(h, C.byref(b), C.byref(p), C.byref(w), C.byref(hh))
    n = b.value * p.value * w.value * hh.value
    out["field32"] = np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64).reshape(
        b.value, p.value, hh.value, w.value)
    L.digHoloDestroy(h)
    return out


@pytest.mark.parametrize("overlap", [0, 1])
@pytest.mark.parametrize("name,inverse", [("square256", 0), ("rect256x128", 0), ("batched128", 2)])
def test_bands_vs_oracle(lib, name, inverse, overlap):
    hol = _case(name)
    cfg = config_for(hol, 0)
    g = _run(lib, hol, cfg, inverse, overlap)
    assert g["kernel"] == 4
    assert g["overlap"] == (2 if overlap == 0 else 1)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert g["R"].shape == o["R"].shape
    np.testing.assert_array_equal(g["x"], o["x"])
    np.testing.assert_array_equal(g["y"], o["y"])
    assert np.max(np.abs(g["scale"].T - o["scale"]) / o["scale"]) <= 1e-5
    assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    err = rel_l2(g["coefs"], o["coefs"])
    print("%s overlap %d: coefficient rel L2 %.2e" % (name, overlap, err))
    assert err <= (1e-4 if overlap == 0 else 5e-5)
    ex = O.process_batch(hol.frames, cfg, quantised=False)
    assert rel_l2(g["field32"], ex["field_v"]) <= 1e-5


def test_bands_match_field_kernel(lib):
    """The 128 x 128 batch through the bands and through the pruned
    full-resolution field kernel: the same int16 fields within 1 LSB and the
    same statistics (batch summary) within FP32 rounding."""
    hol = _case("batched128")
    cfg = config_for(hol, 0)
    a = _run(lib, hol, cfg, 2, 1)
    b = _run(lib, hol, cfg, 0, 1)
    assert b["kernel"] == 3
    assert max(np.abs(a["R"].astype(int) - b["R"]).max(), np.abs(a["I"].astype(int) - b["I"]).max()) <= 1
    np.testing.assert_allclose(a["summary"], b["summary"], rtol=1e-5, atol=1e-6)
    assert rel_l2(a["coefs"], b["coefs"]) <= 1e-5


@pytest.mark.parametrize("name,mode", [("square256", 1), ("rect256x128", 0)])
def test_forward_through_full_planes(lib, name, mode):
    """Windows 256 pixels wide take the full-plane forward path (kernel 5:
    R2C rows, columns, then the window) by default; its Fourier windows agree
    with the generic shared-memory kernel's (kernel 1) within 1e-6 relative
    L2, and with the FP64 oracle's in IFFT mode 1 within 1e-6."""
    hol = _case(name)
    cfg = config_for(hol, mode)
    out = {}
    for fwd in (0, 1):
        h = lib.digHoloCreate()
        api.configure(lib, h, cfg)
        assert lib.digHoloB200SetForwardKernel(h, fwd) == 0
        g = api.run_batch(lib, h, hol.frames)
        assert g["coefs"] is not None, lib.digHoloB200GetLastError(h)
        k = lib.digHoloB200GetForwardKernel(h)
        b, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        wp = lib.digHoloGetFourierPlaneWindow(h, C.byref(b), C.byref(p), C.byref(w), C.byref(hh))
        n = b.value * p.value * w.value * hh.value
        g["window"] = np.ctypeslib.as_array(wp, shape=(2 * n,)).copy().view(np.complex64)
        lib.digHoloDestroy(h)
        out[fwd] = (k, g)
    assert out[0][0] == 5 and out[1][0] == 1
    assert rel_l2(out[0][1]["window"], out[1][1]["window"]) <= 1e-6
    o = O.process_batch(hol.frames, cfg, quantised=True)
    if mode == 1:
        assert rel_l2(out[0][1]["window"], o["window"].ravel()) <= 1e-6
    assert max(np.abs(out[0][1]["R"].astype(int) - o["R"]).max(), np.abs(out[0][1]["I"].astype(int) - o["I"]).max()) <= 2
    assert rel_l2(out[0][1]["coefs"], o["coefs"]) <= 1e-4


NONPOW2 = [
    # frame, FFT window, carrier (fraction of Nyquist), waist -> IFFT window
    ((1280, 1024), (256, 256), (0.38, 0.304), 640e-6, (48, 48)),
    ((640, 512), (128, 128), (0.6, 0.48), 320e-6, (48, 48)),
    ((640, 512), (128, 64), (0.6, 0.48), 320e-6, (48, 32)),
]


@pytest.mark.parametrize("frame,window,carrier,waist,wh", NONPOW2, ids=["256sq_48", "128sq_48", "128x64_48x32"])
@pytest.mark.parametrize("overlap", [0, 1])
def test_non_power_of_two_ifft_window(lib, overlap, frame, window, carrier, waist, wh):
    """Carriers that give IFFT windows whose sides are multiples of 16 but
    not powers of two (48, for FFT windows of 256 and 128 pixels).  At full
    resolution (the reference's default) they run through the full-plane
    forward and the band kernels, which fold any multiple of 16 onto
    16-point transforms: int16 fields within 2 LSB of the quantised oracle,
    coefficients relative L2 <= 1e-4 (split-BF16) or 5e-5 (FP32).  In
    low-resolution mode the field has the window's size and runs through the
    DFT kernel (inverse kernel 6): the same bounds with the FP32 overlap."""
    hol = synth.generate(frame_count=4, frame_width=frame[0], frame_height=frame[1], pol_count=2, max_mg=9, waist=waist,
                         snr_db=30, window=window, dtype="float32", seed=2999, carrier=carrier)
    cfg = config_for(hol, 0)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert (o["w"], o["h"]) == wh
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    assert lib.digHoloB200SetOverlapKernel(h, overlap) == 0
    g = api.run_batch(lib, h, hol.frames)
    assert g["coefs"] is not None, lib.digHoloB200GetLastError(h)
    assert lib.digHoloB200GetForwardKernel(h) == 5 and lib.digHoloB200GetInverseKernel(h) == 4
    assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    assert rel_l2(g["coefs"], o["coefs"]) <= (1e-4 if overlap == 0 else 5e-5)
    cfg1 = config_for(hol, 1)
    api.configure(lib, h, cfg1)
    g1 = api.run_batch(lib, h, hol.frames)
    assert g1["coefs"] is not None, lib.digHoloB200GetLastError(h)
    assert lib.digHoloB200GetForwardKernel(h) == 5 and lib.digHoloB200GetInverseKernel(h) == 6
    o1 = O.process_batch(hol.frames, cfg1, quantised=True)
    assert g1["R"].shape == o1["R"].shape and o1["R"].shape[-2:] == (wh[1], wh[0])
    assert np.max(np.abs(g1["scale"].T - o1["scale"]) / o1["scale"]) <= 1e-5
    assert max(np.abs(g1["R"].astype(int) - o1["R"]).max(), np.abs(g1["I"].astype(int) - o1["I"]).max()) <= 2
    assert rel_l2(g1["field"], o1["field"]) <= 5e-5
    assert rel_l2(g1["coefs"], o1["coefs"]) <= 5e-5
    lib.digHoloDestroy(h)


def test_large_low_resolution_non_power_of_two(lib):
    """A 144 x 144 low-resolution field (FFT windows of 512 pixels, carrier
    (0.6, 0.48) of Nyquist): the DFT kernel's two planes exceed shared memory
    and live in global scratch.  int16 fields within 2 LSB of the quantised
    oracle, scales within 1e-5, fields and coefficients relative L2 <= 5e-5;
    the same with a reference-wave calibration (planes through the same
    kernel)."""
    from helpers import ref_calibration, set_ref_calibration
    hol = synth.generate(frame_count=3, frame_width=1280, frame_height=1024, pol_count=2, max_mg=9, waist=640e-6,
                         snr_db=30, window=(512, 512), dtype="float32", seed=2999, carrier=(0.6, 0.48))
    for calibrated in (False, True):
        cfg = config_for(hol, 1)
        h = lib.digHoloCreate()
        api.configure(lib, h, cfg)
        if calibrated:
            set_ref_calibration(lib, h, cfg, "intensity", ref_calibration(cfg, "intensity"))
        g = api.run_batch(lib, h, hol.frames)
        assert g["coefs"] is not None, lib.digHoloB200GetLastError(h)
        assert lib.digHoloB200GetInverseKernel(h) == 6
        o = O.process_batch(hol.frames, cfg, quantised=True)
        assert o["R"].shape[-2:] == (144, 144) and g["R"].shape == o["R"].shape
        assert np.max(np.abs(g["scale"].T - o["scale"]) / o["scale"]) <= 1e-5
        assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
        assert rel_l2(g["field"], o["field"]) <= 5e-5
        assert rel_l2(g["coefs"], o["coefs"]) <= 5e-5
        lib.digHoloDestroy(h)
