"""digHoloB200ProcessBatchNoAlloc against the regular device entry point.

Some callers cannot allocate device memory while they process frames: a
real-time acquisition callback must not block in cudaMalloc/cudaFree (both
can synchronise the whole device), and some applications fix their memory
pool at start-up.  The no-alloc entry point serves them: the scratch that
carries the Fourier windows from the forward to the inverse kernel is a
static 8 MiB device array, and the caller passes the frames and every output
buffer.  This file runs last (pytest collects it after the others) and
checks the entry point twice in a row against digHoloB200ProcessBatchDevice,
with the coefficient tolerance of the parity tests (relative L2 <= 5e-5) and
identical int16 fields.
"""
import ctypes as C

import numpy as np
import pytest

from digholo_b200 import api
from helpers import config_for, make_case, rel_l2

pytestmark = pytest.mark.gpu


class _DeviceArray:
    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False), "version": 2}


def test_no_alloc_matches_device_entry_point():
    import torch
    import digholo_b200
    L = digholo_b200.load()
    hol = make_case("batched_640x512_u16_2pol", 32)
    cfg = config_for(hol, 1)
    frames = torch.from_numpy(np.ascontiguousarray(hol.frames).view(np.int16)).cuda()
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    B = frames.shape[0]
    fp = C.cast(C.c_void_p(frames.data_ptr()), C.POINTER(C.c_ushort))
    assert L.digHoloSetBatchUint16(h, B, fp, 0) == 0
    assert L.digHoloB200ProcessBatchDevice(h) == 0
    assert L.digHoloB200Synchronize(h) == 0
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    dptr = L.digHoloB200GetCoefsDevice(h, C.byref(b), C.byref(m), C.byref(p))
    assert dptr and m.value == 120 and p.value == 2
    M, P = m.value, p.value
    # the regular entry point leaves the coefficients on the GPU; view them through the CUDA array interface
    dev_view = _DeviceArray(C.cast(dptr, C.c_void_p).value, (B, P * M, 2), "<f4")
    ref_coefs = torch.as_tensor(dev_view, device="cuda").clone()
    geo = (C.c_int * 10)()
    L.digHoloB200GetGeometry(h, geo)
    nx, ny = geo[4], geo[5]
    ref_out = api.read_outputs(L, h, B, want_fields=True)
    for call in range(2):
        coefs = torch.full((B, P * M, 2), float("nan"), dtype=torch.float32, device="cuda")
        fr = torch.full((B, P, ny, nx), 7, dtype=torch.int16, device="cuda")
        fi = torch.full((B, P, ny, nx), 7, dtype=torch.int16, device="cuda")
        stats = torch.zeros((7, P, B + 1), dtype=torch.float32, device="cuda")
        rc = L.digHoloB200ProcessBatchNoAlloc(h, frames.data_ptr(), B, 1, coefs.data_ptr(), fr.data_ptr(),
                                              fi.data_ptr(), stats.data_ptr())
        assert rc == 0, L.digHoloB200GetLastError(h)
        assert L.digHoloB200Synchronize(h) == 0
        got = coefs.cpu().numpy().view(np.complex64).reshape(B, P * M)
        want = ref_coefs.cpu().numpy().view(np.complex64).reshape(B, P * M)
        assert np.isfinite(got).all()
        assert rel_l2(got, want) <= 5e-5
        np.testing.assert_array_equal(fr.cpu().numpy(), ref_out["R"])
        np.testing.assert_array_equal(fi.cpu().numpy(), ref_out["I"])
        np.testing.assert_allclose(stats[3, :, :B].cpu().numpy(), ref_out["scale"], rtol=1e-6)
    # sizes beyond the scratch are refused with an error, not processed
    big = 1 << 20
    rc = L.digHoloB200ProcessBatchNoAlloc(h, frames.data_ptr(), big, 1, coefs.data_ptr(), fr.data_ptr(),
                                          fi.data_ptr(), stats.data_ptr())
    assert rc == 5  # DIGHOLO_ERROR_INVALIDDIMENSION
    L.digHoloDestroy(h)
