"""Transposed uint16 frames (digHoloSetBatchUint16 with transpose = 1).

Each frame is stored with x and y swapped (frameWidth rows of frameHeight
pixels); this build transposes it on the device and processes the result, so
the outputs equal those of the untransposed frames exactly, for square and
non-square frames.  The reference's transposing converter scrambles every
other row (tests/test_reference_defects.py shows it on the reference build),
so there is no reference parity to check for this option.
"""
import ctypes as C

import numpy as np
import pytest

from digholo_b200 import api, synth
from helpers import config_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _run(L, cfg, frames, transpose):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    fr = np.ascontiguousarray(frames)
    assert L.digHoloSetBatchUint16(h, fr.shape[0], fr.ctypes.data_as(C.POINTER(C.c_ushort)), int(transpose)) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    assert cp, L.digHoloB200GetLastError(h)
    out = api.read_outputs(L, h, fr.shape[0], cp, m.value, p.value, True)
    L.digHoloDestroy(h)
    return out


@pytest.mark.parametrize("shape,pols,mode", [((512, 512), 1, 0), ((640, 512), 2, 1)])
def test_transposed_frames_match_plain(lib, shape, pols, mode):
    W, H = shape
    hol = synth.generate(frame_count=4, frame_width=W, frame_height=H, pol_count=pols, max_mg=9, waist=220e-6,
                         snr_db=30, window=(128, 128), dtype="uint16", seed=2024 + W)
    cfg = config_for(hol, mode)
    F = hol.frames                                         # [frame][H][W]
    p = np.ascontiguousarray(np.transpose(F, (0, 2, 1)))   # [frame][W][H]: x and y swapped
    g_plain = _run(lib, cfg, F, 0)
    g_t = _run(lib, cfg, p, 1)
    for k in ("R", "I", "coefs"):
        np.testing.assert_array_equal(g_t[k], g_plain[k])
