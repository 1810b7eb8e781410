"""Auxiliary entry points against the reference build: the basis fields
(digHoloBasisGetFields, digHolo.h:1587) of HG and custom bases, and frames
loaded from a uint16 file (digHoloSetFrameBufferFromFile, digHolo.h:288)
processed like the same frames passed by pointer.

Basis fields: relative L2 <= 1e-6 against the reference (the same int16
modes and float32 accumulation).  Frames from a file: the coefficients equal
those of the pointer path exactly (the same batch); fields and (unscaled
16-row) coefficients within 5e-5 of the reference's.
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


def _basis_fields(L, cfg, frames, custom=None):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    if custom is not None:
        t = np.ascontiguousarray(custom.astype(np.complex64))
        L.digHoloConfigSetBasisTypeCustom(h, t.shape[0], t.shape[1], t.ctypes.data_as(C.POINTER(C.c_float)))
    api.run_batch(L, h, frames, want_fields=False)
    m, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    x, y = C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    fp = L.digHoloBasisGetFields(h, C.byref(m), C.byref(p), C.byref(x), C.byref(y), C.byref(w), C.byref(hh))
    assert fp
    n = m.value * p.value * w.value * hh.value
    return np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64).reshape(m.value, p.value, hh.value,
                                                                                         w.value)


@pytest.mark.parametrize("basis", ["hg", "custom"])
@pytest.mark.parametrize("mode", [1, 0])
def test_basis_fields_match_reference(lib, basis, mode):
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    hol = make_case("batched_640x512_u16_2pol", 2)
    cfg = config_for(hol, mode, max_mg=6)
    custom = None
    if basis == "custom":
        rng = np.random.default_rng(9)
        custom = (rng.standard_normal((21, 12)) + 1j * rng.standard_normal((21, 12))).astype(np.complex64)
    g = _basis_fields(lib, cfg, hol.frames, custom)
    r = _basis_fields(ref_lib.load(), cfg, hol.frames, custom)
    assert g.shape == r.shape
    err = rel_l2(g, r)
    print("%s mode %d basis fields %s: rel L2 %.2e" % (basis, mode, g.shape, err))
    assert err <= 1e-6


def test_frames_from_file(lib, tmp_path):
    hol = make_case("batched_640x512_u16_2pol", 4)
    cfg = config_for(hol, 1)
    path = str(tmp_path / "frames.bin")
    hol.frames.astype(np.uint16).tofile(path)
    out = []
    libs = [lib] + ([ref_lib.load()] if ref_lib.available() else [])
    for L in libs:
        h = L.digHoloCreate()
        api.configure(L, h, cfg)
        L.digHoloConfigSetBatchCount(h, 4)
        assert L.digHoloSetFrameBufferFromFile(h, path.encode()) == 0
        b, m, p = C.c_int(), C.c_int(), C.c_int()
        cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
        assert cp
        out.append(api.read_outputs(L, h, b.value, cp, m.value, p.value, True))
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    ptr = api.run_batch(lib, h, hol.frames.astype(np.float32), want_fields=False)["coefs"]
    assert np.array_equal(out[0]["coefs"], ptr)
    if len(out) > 1:
        g, r = out
        assert rel_l2(g["field"], r["field"]) <= 5e-5
        # the reference leaves the coefficients of 16-row fields unscaled (digHolo.cpp:2318-2331)
        gc = O.reference_unscaled_16(g["coefs"].astype(np.complex128), cfg, {"x": g["x"], "y": g["y"], "scale": g["scale"].T})
        assert rel_l2(gc, r["coefs"]) <= 5e-5
