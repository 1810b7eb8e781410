"""Generates tests/golden/*.npz from the reference build (oracle/_ref).

Each fixture holds the outputs of the unmodified reference's
digHoloProcessBatch on a seeded synthetic hologram: coefficients, int16
fields, field scales and axes.  The frames are not stored: they are
regenerated bit-for-bit by digholo_b200.synth.generate from the stored seed
and parameters (numpy's PCG64 stream is stable).

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import ref_lib  # noqa: E402
from helpers import config_for, make_case  # noqa: E402

CASES = {
    "plain_mode0": ("plain_320x256_f32_1pol", 2, 0),
    "plain_mode1": ("plain_320x256_f32_1pol", 2, 1),
    "dualpol_mode0": ("batched_640x512_u16_2pol", 2, 0),
    "dualpol_mode1": ("batched_640x512_u16_2pol", 2, 1),
}


def main():
    L = ref_lib.load()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, (workload, frames, mode) in CASES.items():
        hol = make_case(workload, frames)
        cfg = config_for(hol, mode)
        h = L.digHoloCreate()
        ref_lib.configure(L, h, cfg)
        r = ref_lib.run_batch(L, h, hol.frames)
        meta = {"workload": workload, "frames": frames, "mode": mode}
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), meta=json.dumps(meta),
                            coefs=r["coefs"], R=r["R"], I=r["I"], scale=r["scale"], x=r["x"], y=r["y"])
        print(name, r["coefs"].shape, r["R"].shape)


if __name__ == "__main__":
    main()
