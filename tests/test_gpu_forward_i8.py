"""Forward stage of uint16 frames on the tensor cores (forward kernel 4):
the row DFT as exact integer tcgen05.mma.kind::i8 products of the frame
bytes with 22-bit fixed-point twiddle digits, then the column stage and the
window factors on the CUDA cores.

Against the FP64 oracle's Fourier window (relative L2 <= 1e-6, the FP32 FFT
kernels reach the same bound) and against the TMA-fed FP32-FFT kernel on the
same frames (relative L2 <= 1e-6); fields and coefficients downstream as in
test_gpu_parity (int16 fields within 2 LSB of the quantised oracle,
coefficients relative L2 <= 5e-5).  Cases: the 640 x 512 two-polarisation
batch (128 x 128 FFT window, 16 x 16 IFFT window) in both IFFT modes, and
carriers at (0.35, 0.3) Nyquist (32 x 32 IFFT window); full 16-bit pixel
values as well as 12-bit ones.
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
    if name == "batched":
        return make_case("batched_640x512_u16_2pol", 16)
    hol = synth.generate(frame_count=16, frame_width=640, frame_height=512, pol_count=2, max_mg=9, waist=220e-6,
                         snr_db=30, window=(128, 128), dtype="uint16", seed=5, carrier=(0.35, 0.3))
    if name == "wide16bit":
        # the full uint16 range: high bytes up to 255
        hol.frames = (hol.frames.astype(np.uint32) * 16 + 7).clip(0, 65535).astype(np.uint16)
    return hol


def _run(L, hol, cfg, fwd):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    assert L.digHoloB200SetForwardKernel(h, fwd) == 0
    out = api.run_batch(L, h, hol.frames)
    assert out["coefs"] is not None, L.digHoloB200GetLastError(h)
    out["fwd"] = L.digHoloB200GetForwardKernel(h)
    b, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    wp = L.digHoloGetFourierPlaneWindow(h, C.byref(b), C.byref(p), C.byref(w), C.byref(hh))
    n = b.value * p.value * w.value * hh.value
    out["window"] = np.ctypeslib.as_array(wp, shape=(2 * n,)).copy().view(np.complex64).reshape(
        b.value, p.value, hh.value, w.value)
    L.digHoloDestroy(h)
    return out


@pytest.mark.parametrize("name,mode", [("batched", 1), ("batched", 0), ("wide", 1), ("wide16bit", 0)])
def test_tensor_core_forward(lib, name, mode):
    hol = _case(name)
    cfg = config_for(hol, mode)
    g = _run(lib, hol, cfg, 0)
    assert g["fwd"] == 4
    t = _run(lib, hol, cfg, 3)
    assert t["fwd"] == 3
    o = O.process_batch(hol.frames, cfg, quantised=True)
    d = rel_l2(g["window"], t["window"])
    if o["window"].shape == g["window"].shape:
        # the oracle keeps the h x w window in IFFT mode 1 (in mode 0 it places it in the H x W plane)
        ew, et = rel_l2(g["window"], o["window"]), rel_l2(t["window"], o["window"])
        print("%s mode %d: window rel L2 tensor-core %.2e, FP32 FFT %.2e; kernel difference %.2e"
              % (name, mode, ew, et, d))
        assert ew <= 1e-6
    else:
        print("%s mode %d: window kernel difference %.2e" % (name, mode, d))
    assert d <= 1e-6
    assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    assert rel_l2(g["coefs"], o["coefs"]) <= (1e-4 if mode == 0 else 5e-5)


@pytest.mark.parametrize("full16", [False, True])
def test_fused_forward_inverse(lib, full16):
    """uint16 frames with 16 x 16 low-resolution fields: forward and inverse
    stages in one launch (inverse choice 3, reported as kernel 5) against the two-launch path
    (tensor-core forward, 64-thread-per-unit inverse; the automatic choice)
    on the same frames.  The fused epilogue runs radix-2 transforms, the
    two-launch inverse a 4 x 4 split, so the two agree to rounding: int16
    fields within 1 step, field scales within 1e-6 relative, coefficients
    within 1e-5 relative L2, and both inside the oracle bounds of
    test_gpu_parity.  12-bit pixels and the full 16-bit range."""
    hol = make_case("batched_640x512_u16_2pol", 16)
    if full16:
        hol.frames = (hol.frames.astype(np.uint32) * 16 + 7).clip(0, 65535).astype(np.uint16)
    cfg = config_for(hol, 1)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    sep = api.run_batch(lib, h, hol.frames)
    ks = (lib.digHoloB200GetForwardKernel(h), lib.digHoloB200GetInverseKernel(h))
    lib.digHoloDestroy(h)
    h2 = lib.digHoloCreate()
    api.configure(lib, h2, cfg)
    assert lib.digHoloB200SetInverseKernel(h2, 3) == 0
    g2 = api.run_batch(lib, h2, hol.frames)
    kf = lib.digHoloB200GetInverseKernel(h2)
    lib.digHoloDestroy(h2)
    assert ks == (4, 2) and kf == 5
    assert np.abs(g2["R"].astype(int) - sep["R"]).max() <= 1
    assert np.abs(g2["I"].astype(int) - sep["I"]).max() <= 1
    assert np.max(np.abs(g2["scale"] - sep["scale"]) / sep["scale"]) <= 1e-6
    d = rel_l2(g2["coefs"], sep["coefs"])
    o = O.process_batch(hol.frames, cfg, quantised=True)
    print("fused vs two launches: coefficient rel L2 %.2e; vs oracle %.2e" % (d, rel_l2(g2["coefs"], o["coefs"])))
    assert d <= 1e-5
    for g in (g2, sep):
        assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
        assert rel_l2(g["coefs"], o["coefs"]) <= 5e-5
