"""The large end of the uneven-batch workload: a 2048-frame batch of
1280x1024 float32 frames (two polarisations, 256x256 FFT windows, maxMG 9,
about 10.7 GB of frames, generated on the GPU with the hologram model of
digholo_b200/synth.py as bench.py does), processed from device memory
between small 320x256 batches on the same handle with the kernel planner
on (FFTW plan mode MEASURE).  Every 128th frame of the large batch, and the
small batches whole, are checked against the oracle at the tolerances of
test_gpu_parity.py (int16 fields within 2 LSB, field relative L2 <= 5e-5,
coefficients relative L2 <= 5e-5); frames are independent, so a frame's
outputs do not depend on the rest of its batch.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
from digholo_b200 import api, synth
from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _cfg(hol, mode):
    return O.Config(frame_width=hol.frame_width, frame_height=hol.frame_height, pixel_size=hol.pixel_size,
                    pol_count=hol.pol_count, fft_window=hol.window, window_radius_deg=hol.radius_deg,
                    resolution_mode=mode, wavelength=hol.wavelength, beam_centre=hol.beam_centres,
                    tilt_deg=hol.tilts_deg, waist=[hol.waist] * 2, max_mg=hol.max_mg)


def _check(g, o, rows):
    dR = np.abs(g["R"].astype(np.int32) - o["R"])
    dI = np.abs(g["I"].astype(np.int32) - o["I"])
    assert max(int(dR.max()), int(dI.max())) <= 2, rows
    assert rel_l2(g["field"], o["field"]) <= 5e-5, rows
    assert rel_l2(g["coefs"], o["coefs"]) <= 5e-5, rows


def _small(lib, h, frames, mg, window, seed):
    hol = synth.generate(frame_count=frames, frame_width=320, frame_height=256, pol_count=2, max_mg=mg,
                         waist=2.5e-6 * window * 2, snr_db=30, window=(window, window), dtype="float32", seed=seed)
    cfg = _cfg(hol, 1)
    api.configure(lib, h, cfg)
    g = api.run_batch(lib, h, hol.frames)
    _check(g, O.process_batch(hol.frames, cfg, quantised=True), "small %d" % frames)


def test_large_batch_between_small_ones(lib):
    import torch
    import bench
    B = 2048
    hol1 = synth.generate(frame_count=1, frame_width=1280, frame_height=1024, pol_count=2, max_mg=9, waist=500e-6,
                          snr_db=30, window=(256, 256), dtype="float32", seed=7001)
    cfg = _cfg(hol1, 1)

    class G:
        pass
    gc = G()
    gc.frame_width, gc.frame_height, gc.pol_count, gc.max_mg = 1280, 1024, 2, 9
    gc.pixel_size, gc.beam_centre, gc.waist = hol1.pixel_size, hol1.beam_centres, [hol1.waist] * 2
    gc.snr_db, gc.taper = 30, False
    dev = bench.torch_frames(gc, B, 7002, torch.device("cuda", 0)).float()   # 12-bit values as float32
    torch.cuda.synchronize()
    assert dev.shape == (B, 1024, 1280)
    h = lib.digHoloCreate()
    assert lib.digHoloConfigSetFFTWPlanMode(h, 1) == 0
    _small(lib, h, 1, 6, 32, 7003)
    api.configure(lib, h, cfg)
    fp = C.cast(C.c_void_p(dev.data_ptr()), C.POINTER(C.c_float))
    assert lib.digHoloSetBatch(h, B, fp) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    assert cp, lib.digHoloB200GetLastError(h)
    g = api.read_outputs(lib, h, B, cp, m.value, p.value, want_fields=True)
    rows = np.arange(0, B, 128)
    sub = dev[torch.as_tensor(rows, device=dev.device)].cpu().numpy()
    o = O.process_batch(sub, cfg, quantised=True)
    gs = {k: g[k][rows] for k in ("R", "I", "field", "coefs")}
    _check(gs, o, "large")
    found = lib.digHoloB200GetKernelPlan(h, None, None, None)
    assert found == 1
    del dev
    torch.cuda.empty_cache()
    _small(lib, h, 777, 15, 64, 7004)
    lib.digHoloDestroy(h)
