"""Uneven streamed batches on one handle (the shape of the uneven-batch
workload): a seeded sequence of batches whose frame count (log-uniform),
frame size (320x256 or 1280x1024 float32), FFT window (64/128 or 128/256
for the small and large frames), carrier (uniform in [0.15, 0.3] Nyquist),
maxMG (6, 9 or 15) and IFFT resolution mode change from one batch to the
next, all processed by the same handle, so every grow-only buffer, cached
tensor map, twiddle-digit table, basis and band scratch is reused or
rebuilt.  Each batch is checked against the oracle (int16 fields within 2
LSB, coefficients relative L2 <= 5e-5, or 1e-4 with the split-BF16
overlap of full-resolution fields).  An IFFT window side that is not a
power of two in low-resolution mode must fail with an error (a documented
limit of this build) and leave the handle usable for the next batch."""
import math

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


def _batches(n, seed=2025):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        big = rng.random() < 0.35
        fw, fh = (1280, 1024) if big else (320, 256)
        frames = int(round(math.exp(rng.uniform(0.0, math.log(24 if big else 160)))))
        window = int(rng.choice([128, 256] if big else [64, 128]))
        c = float(rng.uniform(0.15, 0.3))
        mg = int(rng.choice([6, 9, 15]))
        mode = int(rng.integers(0, 2))
        pols = 2 if (fw // 2 >= window and rng.random() < 0.5) else 1
        out.append(dict(frame_count=frames, frame_width=fw, frame_height=fh, pol_count=pols, max_mg=mg,
                        waist=2.5e-6 * window,
                        snr_db=30, window=(window, window), dtype="float32", seed=3000 + k,
                        carrier=(c, 0.8 * c), mode=mode))
    # a carrier of 0.38 Nyquist with a 256-pixel window: 48 x 48 IFFT window
    out.insert(n // 2, dict(frame_count=3, frame_width=1280, frame_height=1024, pol_count=1, max_mg=9, waist=640e-6,
                            snr_db=30, window=(256, 256), dtype="float32", seed=2999, carrier=(0.38, 0.304), mode=1))
    return out


def test_uneven_batches_on_one_handle(lib):
    h = lib.digHoloCreate()
    checked = rejected = 0
    for spec in _batches(12):
        mode = spec.pop("mode")
        hol = synth.generate(**spec)
        cfg = config_for(hol, mode)
        o = O.process_batch(hol.frames, cfg, quantised=True)
        pow2 = (o["w"] & (o["w"] - 1)) == 0 and (o["h"] & (o["h"] - 1)) == 0
        # other multiples of 16: at full resolution with FFT windows of at least
        # 64 x 64, in low-resolution mode through the DFT kernel
        m16 = o["w"] % 16 == 0 and o["h"] % 16 == 0
        supported = pow2 or (m16 and (mode == 1 or (o["W"] >= 64 and o["H"] >= 64)))
        api.configure(lib, h, cfg)
        g = api.run_batch(lib, h, hol.frames)
        if not supported:
            assert g["coefs"] is None
            assert lib.digHoloB200GetLastError(h)
            rejected += 1
            continue
        assert g["coefs"] is not None, lib.digHoloB200GetLastError(h)
        assert g["R"].shape == o["R"].shape
        assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
        tol = 1e-4 if (mode == 0 and lib.digHoloB200GetOverlapKernel(h) == 2) else 5e-5
        assert rel_l2(g["coefs"], o["coefs"]) <= tol
        checked += 1
    lib.digHoloDestroy(h)
    print("uneven batches: %d checked against the oracle, %d rejected" % (checked, rejected))
    # the 48 x 48 low-resolution batch is among the checked ones
    assert checked >= 7
