"""Forward stage of 512-pixel-wide FFT windows (forward kernel 5, the
full-plane route, automatic for windows of 256 pixels and more).

Two routes, each checked against the oracle (FFTW-equivalent numpy r2c and
digHoloCopyWindow, digHolo.cpp:7184-7260 and 1808-2122) at the tolerances
of test_gpu_parity.py (int16 fields within 2 LSB, field relative L2 <= 5e-5,
coefficients relative L2 <= 5e-5 FP32 / 1e-4 split-BF16):

* 512 x 512 FFT windows with 64 x 64 IFFT windows: register row transform
  (16 x 16 in registers) writing only the window's columns, then the pruned
  64-row column transform with the window factors (dh_plane.cu);
* 512-wide windows whose IFFT window is not 64 rows (48 x 48; 64 x 112 in
  512 x 1024 FFT windows): the register row transform into the plane's layout, then the
  shared-memory column transform and the window copy (dh_fourier.cu).

Frame sides are multiples of 16 pixels (digHoloConfigSetFrameDimensions
refuses others), FFT-window corners multiples of 16 pixels and device frame
buffers 16-byte aligned, so the register row transform's 16-byte loads
always apply; the shared-memory row transform stays behind it for safety.

uint16 and float32 frames, one and two polarisations, both resolution modes,
frames from host memory (the FFT windows staged by a pitched copy) and read
in place from device memory.
"""
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
    # name: (generate kwargs, radius scale, expected (W, H, w, h))
    "w512_f32_1pol_win64": (dict(frame_width=1024, frame_height=1024, pol_count=1, max_mg=15, waist=400e-6,
                                 window=(512, 512), dtype="float32", seed=5101), 1.0, (512, 512, 64, 64)),
    "w512_u16_2pol_win64": (dict(frame_width=1024, frame_height=512, pol_count=2, max_mg=12, waist=350e-6,
                                 window=(512, 512), dtype="uint16", seed=5102), 1.0, (512, 512, 64, 64)),
    "w512_f32_1pol_win48": (dict(frame_width=1024, frame_height=1024, pol_count=1, max_mg=10, waist=400e-6,
                                 window=(512, 512), dtype="float32", seed=5103), 0.7, (512, 512, 48, 48)),
    "w512_h1024_u16_1pol": (dict(frame_width=1024, frame_height=1024, pol_count=1, max_mg=10, waist=400e-6,
                                 window=(512, 1024), dtype="uint16", seed=5104), 1.0, (512, 1024, 64, 112)),
}


def _run(lib, h, frames, device):
    """SetBatch from host memory (the FFT windows staged by a pitched copy)
    or from device memory (the frames read in place), then ProcessBatch."""
    import ctypes as C
    t = None
    if not device:
        rc = api.set_batch(lib, h, frames)
    else:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(frames)).cuda()
        torch.cuda.synchronize()
        if frames.dtype == np.uint16:
            rc = lib.digHoloSetBatchUint16(h, frames.shape[0], C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_ushort)), 0)
        else:
            rc = lib.digHoloSetBatch(h, frames.shape[0], C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float)))
    assert rc == 0
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    assert cp, lib.digHoloB200GetLastError(h)
    out = api.read_outputs(lib, h, frames.shape[0], cp, m.value, pc.value, True)
    del t
    return out


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("mode", [1, 0])
def test_plane512_routes_match_oracle(lib, name, mode, device):
    kw, rscale, geo = CASES[name]
    hol = synth.generate(frame_count=3, snr_db=25, **kw)
    cfg = config_for(hol, mode)
    cfg.window_radius_deg = np.float32(cfg.window_radius_deg * rscale)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    g = _run(lib, h, hol.frames, device)
    assert g["coefs"] is not None, lib.digHoloB200GetLastError(h)
    assert lib.digHoloB200GetForwardKernel(h) == 5
    out = (api.C.c_int * 10)()
    assert lib.digHoloB200GetGeometry(h, out) == 0
    used = lib.digHoloB200GetOverlapKernel(h)
    lib.digHoloDestroy(h)
    assert tuple(out[:4]) == geo
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert g["R"].shape == o["R"].shape
    dmax = max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max())
    ef, ec = rel_l2(g["field"], o["field"]), rel_l2(g["coefs"], o["coefs"])
    print("%s mode %d %s: int16 max diff %d, field rel L2 %.2e, coefs rel L2 %.2e"
          % (name, mode, "device" if device else "host", dmax, ef, ec))
    assert dmax <= 2
    assert ef <= 5e-5
    assert ec <= (1e-4 if used == 2 else 5e-5)
