"""Shared test helpers: build a configuration for a generated hologram and
run it through a library exposing the digHolo C ABI."""
import numpy as np

import digholo_oracle as O
from digholo_b200 import synth


def make_case(workload, frame_count=None, **over):
    kw = dict(synth.WORKLOADS[workload])
    if frame_count is not None:
        kw["frame_count"] = frame_count
    kw.update(over)
    return synth.generate(**kw)


def config_for(hol, mode, max_mg=None):
    return O.Config(frame_width=hol.frame_width, frame_height=hol.frame_height, pixel_size=hol.pixel_size,
                    pol_count=hol.pol_count, fft_window=hol.window, window_radius_deg=hol.radius_deg,
                    resolution_mode=mode, wavelength=hol.wavelength, beam_centre=hol.beam_centres,
                    tilt_deg=hol.tilts_deg, waist=[hol.waist] * 2,
                    max_mg=hol.max_mg if max_mg is None else max_mg)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def ref_calibration(cfg, kind, count=1, seed=3):
    """A reference-wave calibration of the frame's size: uint16 intensities
    of a broad Gaussian beam over a floor with noise, or complex fields with
    ripples in both parts (the reference inverts the parts separately, so
    neither may be zero).  Returns the raw array for the setter."""
    rng = np.random.default_rng(seed)
    fh, fw = cfg.frame_height, cfg.frame_width
    yy, xx = np.mgrid[0:fh, 0:fw]
    if kind == "intensity":
        g = 20000 * np.exp(-((xx - fw / 2) ** 2 + (yy - fh / 2) ** 2) / (2 * (0.4 * fw) ** 2)) + 3000
        return np.stack([g * (1 + 0.1 * c) + rng.integers(0, 200, (fh, fw)) for c in range(count)]).astype(np.uint16)
    return np.stack([(1.0 + 0.3 * np.cos(xx / (37.0 + c)) + 0.2j + 0.1j * np.sin(yy / 23.0)) * np.exp(0.3j * (c + 1))
                     for c in range(count)]).astype(np.complex64)


def set_ref_calibration(L, h, cfg, kind, cal):
    """Apply the calibration through the C ABI and record its stored factors
    in cfg for the oracle."""
    import ctypes as C
    count, fh, fw = cal.shape
    if kind == "intensity":
        r = L.digHoloConfigSetRefCalibrationIntensity(h, cal.ctypes.data_as(C.POINTER(C.c_ushort)), count, fw, fh)
        cfg.ref_cal = O.ref_cal_store(intensity=cal)
    else:
        r = L.digHoloConfigSetRefCalibrationField(h, cal.ctypes.data_as(C.POINTER(C.c_float)), count, fw, fh)
        cfg.ref_cal = O.ref_cal_store(field=cal)
    assert r == 0


def ref_calibration_planes(L, h):
    """digHoloConfigGetRefCalibrationFields as (count, pol, height, width)
    complex64, or None."""
    import ctypes as C
    n, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    x, y = C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    ptr = L.digHoloConfigGetRefCalibrationFields(h, C.byref(n), C.byref(p), C.byref(x), C.byref(y), C.byref(w),
                                                  C.byref(hh))
    if not ptr:
        return None
    N = n.value * p.value * w.value * hh.value
    a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(2 * N,)).copy().view(np.complex64)
    return a.reshape(n.value, p.value, hh.value, w.value)


def reference_calibrated(workload, frames, mode, kind, count, window=None, sweep=None, tries=2):
    """The reference build's batch with a reference-wave calibration, run in
    a child process (refcal_child.py): the reference's calibrated batches
    occasionally corrupt its heap, so they never run in the test process.  A
    child that dies is run once more; its outputs are used only when it
    completed."""
    import os
    import subprocess
    import sys
    import tempfile
    child = os.path.join(os.path.dirname(os.path.abspath(__file__)), "refcal_child.py")
    args = [str(workload), str(frames), str(mode), kind, str(count), str(window) if window else "-",
            ",".join("%.6e" % v for v in sweep) if sweep else "-"]
    last = ""
    for _ in range(tries):
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "r.npz")
            r = subprocess.run([sys.executable, child, out] + args, capture_output=True, text=True, timeout=900)
            if r.returncode == 0 and os.path.exists(out):
                z = np.load(out)
                return {k: z[k] for k in z.files}
            last = (r.stdout + r.stderr)[-2000:]
    raise RuntimeError("reference child process failed: " + last)
