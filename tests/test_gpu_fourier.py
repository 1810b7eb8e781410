"""The Fourier plane of the camera (digHoloGetFourierPlaneFull) and its
analysis (digHoloBatchGetSummary, plane 0), computed on request from the
last batch's frames, against the oracle (which is pinned to the reference in
tests/test_oracle_pin.py): plane relative L2 <= 1e-6, statistics relative
<= 1e-4, the maximum's index equal, batch-sum plane relative L2 <= 1e-5.
Host and device frames, uint16 and float32, one and two polarisations."""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
from digholo_b200 import api
from helpers import config_for, make_case, rel_l2
from test_oracle_pin import check_fourier

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


@pytest.mark.parametrize("workload,device", [("plain_320x256_f32_1pol", False), ("batched_640x512_u16_2pol", False),
                                             ("batched_640x512_u16_2pol", True)])
def test_fourier_plane_and_analysis(lib, workload, device):
    hol = make_case(workload, 6)
    cfg = config_for(hol, 1)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    if device:
        torch = pytest.importorskip("torch")
        t = torch.from_numpy(np.ascontiguousarray(hol.frames).view(np.int16)).cuda()
        lib.digHoloSetBatchUint16(h, t.shape[0], C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_ushort)), 0)
        b, m, p = C.c_int(), C.c_int(), C.c_int()
        assert lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    else:
        api.run_batch(lib, h, hol.frames)
    f = api.read_fourier(lib, h)
    lib.digHoloDestroy(h)
    assert f["summary_rc"] == 0
    o = O.process_batch(hol.frames, cfg, quantised=True)
    check_fourier(o, f, cfg)
