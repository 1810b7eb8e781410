"""Batches of frames at several wavelengths (digHoloProcessBatchFrequencySweepLinear,
digHoloProcessBatchWavelengthSweepArbitrary, digHolo.h:1510-1525, with the
orderings of digHoloConfigSetWavelengthOrdering, digHolo.h:886): against
the reference build on the same frames, settings and orderings.

Each wavelength's frames have their own Fourier-window mask and centre
(k0 of that wavelength) and reference wave, inside the IFFT window that
spans the first and last wavelength.  Checked: the wavelength array
GetWavelengths returns after processing (float32, exactly), int16 fields
within 2 LSB, fields relative L2 <= 5e-5, coefficients relative L2 <= 5e-5,
for wavelength-fast and wavelength-slow input and output orderings, one
and two polarisations.
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
    ("plain_320x256_f32_1pol", 8, (1540e-9, 1590e-9, 4), (0, 1)),
    ("plain_320x256_f32_1pol", 8, (1540e-9, 1590e-9, 4), (1, 0)),
    ("batched_640x512_u16_2pol", 6, [1550e-9, 1575e-9, 1600e-9], (1, 1)),
    ("batched_640x512_u16_2pol", 6, [1550e-9, 1600e-9], (0, 1)),
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
    ef, ec = rel_l2(g["field"], r["field"]), rel_l2(g["coefs"], r["coefs"])
    print("%s %s %s: int16 max diff %d, field rel L2 %.2e, coefs rel L2 %.2e" % (workload, lams, ordering, dmax, ef, ec))
    assert dmax <= 2
    assert ef <= 5e-5
    assert ec <= 5e-5


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
