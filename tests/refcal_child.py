"""Runs one reference-build batch with a reference-wave calibration in its own
process and saves the outputs to an .npz file.

The reference's calibrated batches occasionally leave its heap corrupted
(glibc aborts later allocations in the same process, non-deterministically),
so the tests call the reference's calibration path through this child
process and keep their own process clean.

Usage: python refcal_child.py OUT.npz WORKLOAD FRAMES MODE KIND COUNT [WINDOW|-] [SWEEP|-]
WINDOW: FFT window side (e.g. 256); SWEEP: comma-separated wavelengths.
"""
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(ROOT, "oracle"), ROOT]

import numpy as np  # noqa: E402

import ref_lib  # noqa: E402
from digholo_b200 import api  # noqa: E402
from helpers import config_for, make_case, ref_calibration, ref_calibration_planes, set_ref_calibration  # noqa: E402


def main(argv):
    out, workload, frames, mode, kind, count = argv[:6]
    window = argv[6] if len(argv) > 6 and argv[6] != "-" else None
    sweep = argv[7] if len(argv) > 7 and argv[7] != "-" else None
    hol = make_case(workload, int(frames))
    cfg = config_for(hol, int(mode))
    if window:
        cfg.fft_window = (int(window), int(window))
    cal = ref_calibration(cfg, kind, int(count))
    L = ref_lib.load()
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    set_ref_calibration(L, h, cfg, kind, cal)
    # the library keeps only the pointer: the array must outlive the processing
    fr = np.ascontiguousarray(hol.frames if hol.frames.dtype == np.uint16 else hol.frames.astype(np.float32))
    assert api.set_batch(L, h, fr) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    if sweep:
        lams = [float(v) for v in sweep.split(",")]
        arr = (C.c_float * len(lams))(*lams)
        cp = L.digHoloProcessBatchWavelengthSweepArbitrary(h, C.byref(b), C.byref(m), C.byref(p), arr, len(lams))
    else:
        cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    assert cp
    r = api.read_outputs(L, h, fr.shape[0], cp, m.value, p.value, True)
    planes = ref_calibration_planes(L, h)
    keep = {k: v for k, v in r.items() if isinstance(v, np.ndarray)}
    if planes is not None:
        keep["planes"] = planes
    np.savez(out, **keep)
    sys.stdout.flush()
    os._exit(0)   # skip the reference's teardown


if __name__ == "__main__":
    main(sys.argv[1:])
