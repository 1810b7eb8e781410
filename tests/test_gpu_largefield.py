"""Large-field batches: 2048 x 2048 uint16 frames, two polarisations, FFT
window 512 x 512 (IFFT window 64 x 64), maxMG 30 (465 modes), waist 600 um,
20 dB SNR, 1/(group + 1) amplitude taper; both IFFT resolution modes, a few
frames.  In mode 0 the 512 x 512 fields take the band kernels, with the
overlap exact in integers on the tensor cores and in FP32 on the CUDA cores,
each scored against the FP64 overlap of the same int16 fields (the quantised
oracle) with the worst mode group printed.  Tolerances as in
test_gpu_parity: int16 fields within 2 LSB of the quantised oracle, field
relative L2 <= 5e-5, coefficients relative L2 <= 5e-5 (FP32) or 1e-4
(split-BF16); the reference build agrees within the same bounds.
"""
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


@pytest.fixture(scope="module")
def hol():
    return make_case("largefield_2048_u16_2pol", 2)


def _per_group(c, co, G):
    c, co = c.reshape(-1, c.shape[-1]), co.reshape(-1, co.shape[-1])
    per, s = [], 0
    for grp in range(G):
        sl = slice(s, s + grp + 1)
        per.append(float(np.linalg.norm(c[:, sl] - co[:, sl]) / np.linalg.norm(co[:, sl])))
        s += grp + 1
    return np.array(per)


@pytest.mark.parametrize("mode,overlap,max_mg", [(1, 0, None), (0, 0, None), (0, 1, None), (0, 0, 34)])
def test_largefield_vs_oracle_and_reference(lib, hol, mode, overlap, max_mg):
    """maxMG 34 (595 modes) exceeds the band kernels' 32-group overlap
    tiles: the band pass writes the fields, the chunked FP32 overlap reads
    them."""
    cfg = config_for(hol, mode, max_mg=max_mg)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    assert lib.digHoloB200SetOverlapKernel(h, overlap) == 0
    g = api.run_batch(lib, h, hol.frames)
    assert g["coefs"] is not None, lib.digHoloB200GetLastError(h)
    kern, used = lib.digHoloB200GetInverseKernel(h), lib.digHoloB200GetOverlapKernel(h)
    lib.digHoloDestroy(h)
    if mode == 0 and max_mg:
        assert used == 1   # FP32 (chunked)
    elif mode == 0:
        # tensor cores: the 64-point band kernel with the exact integer overlap
        assert (kern, used) == ((7, 3) if overlap == 0 else (4, 1))
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert g["R"].shape == o["R"].shape
    assert max(np.abs(g["R"].astype(int) - o["R"]).max(), np.abs(g["I"].astype(int) - o["I"]).max()) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    err = rel_l2(g["coefs"], o["coefs"])
    per = _per_group(g["coefs"], o["coefs"], cfg.max_mg)
    print("mode %d %s overlap: coefficient rel L2 %.2e, worst mode group %.2e (group %d)"
          % (mode, {2: "split-BF16", 3: "integer"}.get(used, "FP32"), err, per.max(), int(per.argmax())))
    assert err <= (1e-4 if used == 2 else 5e-5)
    if ref_lib.available():
        L = ref_lib.load()
        hr = L.digHoloCreate()
        ref_lib.configure(L, hr, cfg)
        r = ref_lib.run_batch(L, hr, hol.frames)
        assert rel_l2(g["field"], r["field"]) <= 5e-5
        assert rel_l2(g["coefs"], r["coefs"]) <= (1e-4 if used == 2 else 5e-5)
