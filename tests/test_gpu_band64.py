"""Full-resolution fields 512 pixels wide with IFFT windows up to 64 x 64
(inverse kernel 7, dh_band64.cu): 64-point sub-transforms on lane quads, a
statistics pass and a quantising pass, and the overlap as an exact integer
contraction (byte-split int16 x int16 on the tensor cores, overlap kernel 3).

Checked against the oracle at the tolerances of test_gpu_parity.py: int16
fields within 2 LSB of the quantised oracle, field relative L2 <= 5e-5,
scales relative <= 1e-5, FP32 fields before rounding relative L2 <= 1e-5
against the unquantised oracle; coefficients relative L2 <= 5e-5 (the
integer contraction is exact, so the FP64 oracle bound of the FP32 kernel
applies).  Cases: 512 x 512 FFT windows with 64 x 64 and 48 x 48 IFFT
windows, a 512 x 256 FFT window (32-row IFFT window, four bands), mode
groups up to 16 and above (16- and 32-row Hx operands), no overlap
(maxMG 0), and the FP32 overlap choice, which keeps the older band kernels.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
from digholo_b200 import api, synth
from helpers import config_for, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


CASES = {
    # name: generate kwargs, radius scale, maxMG override
    "sq512_win64_mg15": (dict(frame_width=1024, frame_height=512, pol_count=2, max_mg=15, waist=350e-6,
                              window=(512, 512), dtype="uint16", seed=6101), 1.0, None),
    "sq512_win64_mg8": (dict(frame_width=512, frame_height=512, pol_count=1, max_mg=8, waist=300e-6,
                             window=(512, 512), dtype="float32", seed=6102), 1.0, None),
    "sq512_win48_mg12": (dict(frame_width=512, frame_height=512, pol_count=1, max_mg=12, waist=350e-6,
                              window=(512, 512), dtype="float32", seed=6103), 0.7, None),
    "w512h256_mg10": (dict(frame_width=1024, frame_height=256, pol_count=2, max_mg=10, waist=250e-6,
                           window=(512, 256), dtype="uint16", seed=6104), 1.0, None),
    "sq512_no_overlap": (dict(frame_width=512, frame_height=512, pol_count=1, max_mg=6, waist=300e-6,
                              window=(512, 512), dtype="float32", seed=6105), 1.0, 0),
}


def _run(lib, hol, cfg, overlap):
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    assert lib.digHoloB200SetOverlapKernel(h, overlap) == 0
    lib.digHoloB200SetKeepField32(h, 1)
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    assert api.set_batch(lib, h, hol.frames) == 0
    cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    assert cp or cfg.max_mg == 0, lib.digHoloB200GetLastError(h)
    out = api.read_outputs(lib, h, hol.frames.shape[0], cp, m.value, pc.value, True)
    out["kernel"] = lib.digHoloB200GetInverseKernel(h)
    out["overlap"] = lib.digHoloB200GetOverlapKernel(h)
    bb, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    fp = lib.digHoloB200GetFields32(h, C.byref(bb), C.byref(p), C.byref(w), C.byref(hh))
    n = bb.value * p.value * w.value * hh.value
    out["field32"] = np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64).reshape(
        bb.value, p.value, hh.value, w.value)
    lib.digHoloDestroy(h)
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_band64_vs_oracle(lib, name):
    kw, rscale, mg = CASES[name]
    hol = synth.generate(frame_count=5, snr_db=25, **kw)
    cfg = config_for(hol, 0, max_mg=mg)
    cfg.window_radius_deg = np.float32(cfg.window_radius_deg * rscale)
    g = _run(lib, hol, cfg, 0)
    assert g["kernel"] == 7
    assert g["overlap"] == (3 if cfg.max_mg > 0 else 0)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert g["R"].shape == o["R"].shape
    np.testing.assert_array_equal(g["x"], o["x"])
    np.testing.assert_array_equal(g["y"], o["y"])
    assert np.max(np.abs(g["scale"].T - o["scale"]) / o["scale"]) <= 1e-5
    dmax = max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max())
    ef = rel_l2(g["field"], o["field"])
    msg = "%s: int16 max diff %d, field rel L2 %.2e" % (name, dmax, ef)
    if cfg.max_mg > 0:
        ec = rel_l2(g["coefs"], o["coefs"])
        msg += ", coefs rel L2 %.2e" % ec
        assert ec <= 5e-5
    print(msg)
    assert dmax <= 2
    assert ef <= 5e-5
    ex = O.process_batch(hol.frames, cfg, quantised=False)
    assert rel_l2(g["field32"], ex["field_v"]) <= 1e-5


def test_band64_matches_older_bands(lib):
    """The same batch through the integer overlap (kernel 7) and the FP32
    overlap (which keeps the older band kernels, kernel 4): int16 fields
    within 1 LSB, statistics within FP32 rounding, coefficients within 2e-5."""
    kw, _, _ = CASES["sq512_win64_mg15"]
    hol = synth.generate(frame_count=3, snr_db=25, **kw)
    cfg = config_for(hol, 0)
    a = _run(lib, hol, cfg, 0)
    b = _run(lib, hol, cfg, 1)
    assert a["kernel"] == 7 and b["kernel"] == 4 and b["overlap"] == 1
    assert max(np.abs(a["R"].astype(int) - b["R"]).max(), np.abs(a["I"].astype(int) - b["I"]).max()) <= 1
    np.testing.assert_allclose(a["summary"], b["summary"], rtol=1e-5, atol=1e-6)
    assert rel_l2(a["coefs"], b["coefs"]) <= 2e-5
