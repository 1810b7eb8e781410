"""GPU parity of frame averaging (digHoloSetBatchAvg / digHoloSetBatchAvgUint16,
digHolo.cpp:4401-4463 and the averaging branch of the window copy,
digHolo.cpp:1886-2118, 8636-8672): batchCount x avgCount frames in, batchCount
phase-aligned averaged windows, fields and coefficients out, against the
oracle's average_windows.

Tolerances are those of the plain batch path: int16 fields within 2 LSB,
field scales relative <= 1e-5, complex fields and coefficients relative
L2 <= 5e-5 (1e-4 for the split-BF16 tensor-core overlap of full-resolution
fields).
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
from digholo_b200 import api
from helpers import config_for, make_case, rel_l2

pytestmark = pytest.mark.gpu

AVG = 3


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _run_avg(lib, cfg, frames, avg, mode):
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    frames = np.ascontiguousarray(frames if frames.dtype == np.uint16 else frames.astype(np.float32))
    B = frames.shape[0] // avg
    assert api.set_batch_avg(lib, h, frames, avg, mode) == 0
    if mode == 2:   # the float setter folds mode 2 to 0, as the reference does
        assert lib.digHoloConfigSetBatchAvgMode(h, 2) == 0
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    assert b.value == B
    out = api.read_outputs(lib, h, B, cp, m.value, pc.value, True)
    out["avg_mode"] = lib.digHoloConfigGetBatchAvgMode(h)
    out["overlap"] = lib.digHoloB200GetOverlapKernel(h)
    out["summary_count"] = out["summary"].shape[-1]
    lib.digHoloDestroy(h)
    return out


CASES = [
    ("plain_320x256_f32_1pol", 12, 1, 0),
    ("plain_320x256_f32_1pol", 12, 1, 1),
    ("plain_320x256_f32_1pol", 12, 0, 1),
    ("batched_640x512_u16_2pol", 12, 1, 0),
    ("batched_640x512_u16_2pol", 12, 1, 2),
    ("batched_640x512_u16_2pol", 12, 0, 1),
]


@pytest.mark.parametrize("workload,frames,res_mode,avg_mode", CASES)
def test_averaged_batch_vs_oracle(lib, workload, frames, res_mode, avg_mode):
    hol = make_case(workload, frames)
    cfg = config_for(hol, res_mode)
    cfg.avg_count, cfg.avg_mode = AVG, avg_mode
    g = _run_avg(lib, cfg, hol.frames, AVG, avg_mode)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    B = frames // AVG
    assert g["avg_mode"] == avg_mode
    assert g["R"].shape == o["R"].shape and g["R"].shape[0] == B
    # the summary keeps the reference's batch x avg + 1 entries per polarisation
    assert g["summary_count"] == B * AVG + 1
    np.testing.assert_array_equal(g["x"], o["x"])
    np.testing.assert_array_equal(g["y"], o["y"])
    assert np.max(np.abs(g["scale"].T - o["scale"]) / o["scale"]) <= 1e-5
    dR = np.abs(g["R"].astype(int) - o["R"])
    dI = np.abs(g["I"].astype(int) - o["I"])
    assert max(dR.max(), dI.max()) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    assert rel_l2(g["coefs"], o["coefs"]) <= (1e-4 if g["overlap"] == 2 else 5e-5)


def test_average_of_identical_frames_is_the_frame(lib):
    """avgCount copies of each frame (interlaced) average to the frame itself:
    the aligned phase of a window against itself is 1."""
    hol = make_case("batched_640x512_u16_2pol", 4)
    cfg = config_for(hol, 1)
    one = _run_avg(lib, cfg, hol.frames, 1, 0)
    rep = np.concatenate([hol.frames] * AVG, axis=0)
    cfg.avg_count, cfg.avg_mode = AVG, 1
    g = _run_avg(lib, cfg, rep, AVG, 1)
    assert rel_l2(g["field"], one["field"]) <= 1e-5
    assert rel_l2(g["coefs"], one["coefs"]) <= 1e-5


@pytest.mark.parametrize("avg", [1, 3])
def test_batch_calibration_vs_oracle(lib, avg):
    """Batch calibration (one complex factor per polarisation and batch
    item, cycled over the batch, digHolo.cpp:1831-1835, 2007-2008, 8636-8641)
    without and with frame averaging, against the oracle."""
    hol = make_case("batched_640x512_u16_2pol", 4 * avg)
    cfg = config_for(hol, 1)
    rng = np.random.default_rng(7)
    cfg.batch_cal = rng.uniform(0.5, 2.0, (2, 3)) * np.exp(1j * rng.uniform(-np.pi, np.pi, (2, 3)))
    cfg.avg_count, cfg.avg_mode = avg, 0
    g = _run_avg(lib, cfg, hol.frames, avg, 0)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert np.max(np.abs(g["scale"].T - o["scale"]) / o["scale"]) <= 1e-5
    dR = np.abs(g["R"].astype(int) - o["R"])
    dI = np.abs(g["I"].astype(int) - o["I"])
    assert max(dR.max(), dI.max()) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    assert rel_l2(g["coefs"], o["coefs"]) <= 5e-5
