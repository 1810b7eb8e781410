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
