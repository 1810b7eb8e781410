"""Batches of frames at several wavelengths (digHoloProcessBatchFrequencySweepLinear,
digHoloProcessBatchWavelengthSweepArbitrary, digHolo.h:1510-1525, with the
orderings of digHoloConfigSetWavelengthOrdering, digHolo.h:886): against
the reference build on the same frames, settings and orderings.

Each wavelength's frames have their own Fourier-window mask and centre
(k0 of that wavelength) and reference wave, inside the IFFT window that
spans the first and last wavelength.  Checked against the reference with the
same input and output ordering (wavelength fast, or slow): the wavelength
array GetWavelengths returns after processing (float32, exactly), int16
fields within 2 LSB, fields relative L2 <= 5e-5, coefficients relative L2
<= 5e-5 (with the reference's unscaled coefficients of 16-row fields,
digHolo.cpp:2318-2331, as in test_gpu_parity), one and two polarisations.

With different input and output orderings the reference picks the
reference wave of each output slot as if the slot were an input index
(applyTilt16, digHolo.cpp:2752-2764), i.e. the wave of another wavelength.
This build uses each frame's own wavelength; those orderings are checked as
the permutation of the same-ordering outputs that they are.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
import ref_lib
from digholo_b200 import api
from helpers import config_for, make_case, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _sweep(L, cfg, frames, ordering, lams):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    L.digHoloConfigSetWavelengthOrdering(h, 0, ordering[0])
    L.digHoloConfigSetWavelengthOrdering(h, 1, ordering[1])
    assert api.set_batch(L, h, frames) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    if isinstance(lams, tuple):
        cp = L.digHoloProcessBatchFrequencySweepLinear(h, C.byref(b), C.byref(m), C.byref(p), lams[0], lams[1], lams[2])
    else:
        arr = (C.c_float * len(lams))(*lams)
        cp = L.digHoloProcessBatchWavelengthSweepArbitrary(h, C.byref(b), C.byref(m), C.byref(p), arr, len(lams))
    assert cp
    out = api.read_outputs(L, h, frames.shape[0], cp, m.value, p.value, True)
    n = C.c_int()
    wp = L.digHoloConfigGetWavelengths(h, C.byref(n))
    out["lams"] = np.ctypeslib.as_array(wp, shape=(n.value,)).copy()
    return out


CASES = [
    ("plain_320x256_f32_1pol", 8, (1540e-9, 1590e-9, 4), (0, 0)),
    ("plain_320x256_f32_1pol", 8, (1540e-9, 1590e-9, 4), (1, 1)),
    ("batched_640x512_u16_2pol", 6, [1550e-9, 1575e-9, 1600e-9], (1, 1)),
    ("batched_640x512_u16_2pol", 6, [1550e-9, 1600e-9], (0, 0)),
]


@pytest.mark.parametrize("workload,frames,lams,ordering", CASES, ids=[str(i) for i in range(len(CASES))])
def test_sweep_matches_reference(lib, workload, frames, lams, ordering):
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    hol = make_case(workload, frames)
    cfg = config_for(hol, 1)
    g = _sweep(lib, cfg, hol.frames, ordering, lams)
    r = _sweep(ref_lib.load(), cfg, hol.frames, ordering, lams)
    np.testing.assert_array_equal(g["lams"], r["lams"])
    assert g["R"].shape == r["R"].shape
    dmax = max(np.abs(g["R"].astype(int) - r["R"]).max(), np.abs(g["I"].astype(int) - r["I"]).max())
    gc = g["coefs"]
    if cfg.resolution_mode == 1 and g["R"].shape[-2] == 16:
        gc = O.reference_unscaled_16(gc.astype(np.complex128), cfg, {"x": g["x"], "y": g["y"], "scale": g["scale"].T})
    ef, ec = rel_l2(g["field"], r["field"]), rel_l2(gc, r["coefs"])
    print("%s %s %s: int16 max diff %d, field rel L2 %.2e, coefs rel L2 %.2e" % (workload, lams, ordering, dmax, ef, ec))
    assert dmax <= 2
    assert ef <= 5e-5
    assert ec <= 5e-5


@pytest.mark.parametrize("ordering", [(0, 1), (1, 0)])
def test_mixed_orderings_permute_outputs(lib, ordering):
    hol = make_case("batched_640x512_u16_2pol", 6)
    cfg = config_for(hol, 1)
    lams = [1550e-9, 1575e-9, 1600e-9]
    L, B = 3, 6
    S = B // L
    same = _sweep(lib, cfg, hol.frames, (ordering[0], ordering[0]), lams)
    mixed = _sweep(lib, cfg, hol.frames, ordering, lams)
    for i in range(B):
        if ordering[0] == 0:   # wavelength fast in: frame i -> slow out slot
            lam, sub = i % L, i // L
            a, b = lam * S + sub, i
        else:                  # wavelength slow in: frame i -> fast out slot
            lam, sub = i // S, i % S
            a, b = sub * L + lam, i
        assert np.array_equal(mixed["R"][a], same["R"][b]) and np.array_equal(mixed["I"][a], same["I"][b])
        assert np.array_equal(mixed["coefs"][a], same["coefs"][b])


def test_single_wavelength_sweep_is_the_centre_wavelength(lib):
    """A sweep of one wavelength processes at the centre wavelength
    (digHolo.cpp:7852-7860): the same outputs as ProcessBatch, and the
    oracle's."""
    hol = make_case("plain_320x256_f32_1pol", 4)
    cfg = config_for(hol, 1)
    g = _sweep(lib, cfg, hol.frames, (0, 0), [1500e-9])
    assert np.array_equal(g["lams"], np.array([cfg.wavelength], dtype=np.float32))
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
    assert rel_l2(g["coefs"], o["coefs"]) <= 5e-5


@pytest.mark.parametrize("avg_mode", [0, 1, 2])
def test_sweep_with_frame_averaging_matches_reference(lib, avg_mode):
    """Frame averaging within a multi-wavelength batch: each item's frames
    are those of the reference's averaging modes (digHolo.cpp:8661-8672:
    item b's k-th frame at b A + k, k B + b or b + k L), averaged with the
    phase alignment and processed at the item's wavelength.  Against the
    reference build on the same frames: int16 fields within 2 LSB, fields
    and (unscaled 16-row) coefficients relative L2 <= 5e-5."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    A, B = 2, 6
    hol = make_case("batched_640x512_u16_2pol", A * B)
    cfg = config_for(hol, 1)
    lams = [1550e-9, 1575e-9, 1600e-9]
    out = []
    for L in (lib, ref_lib.load()):
        h = L.digHoloCreate()
        api.configure(L, h, cfg)
        frames = np.ascontiguousarray(hol.frames)
        assert api.set_batch_avg(L, h, frames, A, avg_mode) == 0
        b, m, p = C.c_int(), C.c_int(), C.c_int()
        arr = (C.c_float * 3)(*lams)
        cp = L.digHoloProcessBatchWavelengthSweepArbitrary(h, C.byref(b), C.byref(m), C.byref(p), arr, 3)
        assert cp, (L.digHoloB200GetLastError(h) if hasattr(L, "digHoloB200GetLastError") else "")
        out.append(api.read_outputs(L, h, B, cp, m.value, p.value, True))
    g, r = out
    dmax = max(np.abs(g["R"].astype(int) - r["R"]).max(), np.abs(g["I"].astype(int) - r["I"]).max())
    gc = O.reference_unscaled_16(g["coefs"].astype(np.complex128), cfg, {"x": g["x"], "y": g["y"], "scale": g["scale"].T})
    print("avg mode %d: int16 max diff %d, fields %.2e, coefs %.2e" % (avg_mode, dmax, rel_l2(g["field"], r["field"]),
                                                                      rel_l2(gc, r["coefs"])))
    assert dmax <= 2
    assert rel_l2(g["field"], r["field"]) <= 5e-5
    assert rel_l2(gc, r["coefs"]) <= 5e-5
