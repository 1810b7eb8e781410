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
identical int16 fields: once with 16x16 low-resolution fields, once with
large fields (2048x2048 frames, 512x512 windows: the full-plane forward and
the band inverse, whose scratch buffers the preparing batch sized).  Free
device memory is read before and after every call but the first (the first
call on a device looks up the static scratch array there, and CUDA's lazy
module loading places the 8 MiB array in device memory at that moment): an
allocation by the entry point would show.
A call with more frames than the preparing batch on the large-field
configuration is refused (DIGHOLO_ERROR_MEMORYALLOCATION), not allocated.
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


CASES = [("batched_640x512_u16_2pol", 32, 1, 16), ("largefield_2048_u16_2pol", 4, 0, 2)]


@pytest.mark.parametrize("workload,frames,mode,smaller", CASES)
def test_no_alloc_matches_device_entry_point(workload, frames, mode, smaller):
    import torch
    import digholo_b200
    L = digholo_b200.load()
    hol = make_case(workload, frames)
    cfg = config_for(hol, mode)
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
    G = hol.max_mg
    assert dptr and m.value == G * (G + 1) // 2 and p.value == 2
    M, P = m.value, p.value
    # the regular entry point leaves the coefficients on the GPU; view them through the CUDA array interface
    dev_view = _DeviceArray(C.cast(dptr, C.c_void_p).value, (B, P * M, 2), "<f4")
    ref_coefs = torch.as_tensor(dev_view, device="cuda").clone()
    geo = (C.c_int * 10)()
    L.digHoloB200GetGeometry(h, geo)
    nx, ny = geo[4], geo[5]
    ref_out = api.read_outputs(L, h, B, want_fields=True)
    want_all = ref_coefs.cpu().numpy().view(np.complex64).reshape(B, P * M)
    # the full batch twice, then a smaller one (the leading frames)
    for call, n in enumerate((B, B, smaller)):
        coefs = torch.full((n, P * M, 2), float("nan"), dtype=torch.float32, device="cuda")
        fr = torch.full((n, P, ny, nx), 7, dtype=torch.int16, device="cuda")
        fi = torch.full((n, P, ny, nx), 7, dtype=torch.int16, device="cuda")
        stats = torch.zeros((7, P, n + 1), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.digHoloB200ProcessBatchNoAlloc(h, frames.data_ptr(), n, 1, coefs.data_ptr(), fr.data_ptr(),
                                              fi.data_ptr(), stats.data_ptr())
        assert rc == 0, L.digHoloB200GetLastError(h)
        assert L.digHoloB200Synchronize(h) == 0
        if call > 0:
            assert torch.cuda.mem_get_info()[0] >= free0      # nothing was allocated
        got = coefs.cpu().numpy().view(np.complex64).reshape(n, P * M)
        assert np.isfinite(got).all()
        assert rel_l2(got, want_all[:n]) <= 5e-5
        np.testing.assert_array_equal(fr.cpu().numpy(), ref_out["R"][:n])
        np.testing.assert_array_equal(fi.cpu().numpy(), ref_out["I"][:n])
        np.testing.assert_allclose(stats[3, :, :n].cpu().numpy(), ref_out["scale"][:, :n], rtol=1e-6)
    if mode == 0:
        # more frames than the preparing batch: its plane and band buffers are
        # too small, and the call is refused instead of growing them
        big = torch.cat([frames, frames])
        n = big.shape[0]
        coefs = torch.zeros((n, P * M, 2), dtype=torch.float32, device="cuda")
        fr = torch.zeros((n, P, ny, nx), dtype=torch.int16, device="cuda")
        fi = torch.zeros((n, P, ny, nx), dtype=torch.int16, device="cuda")
        stats = torch.zeros((7, P, n + 1), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.digHoloB200ProcessBatchNoAlloc(h, big.data_ptr(), n, 1, coefs.data_ptr(), fr.data_ptr(),
                                              fi.data_ptr(), stats.data_ptr())
        assert rc == 9, rc  # DIGHOLO_ERROR_MEMORYALLOCATION
        assert L.digHoloB200Synchronize(h) == 0
        assert torch.cuda.mem_get_info()[0] >= free0
    # sizes beyond the scratch are refused with an error, not processed
    big = 1 << 20
    rc = L.digHoloB200ProcessBatchNoAlloc(h, frames.data_ptr(), big, 1, coefs.data_ptr(), fr.data_ptr(),
                                          fi.data_ptr(), stats.data_ptr())
    assert rc == 5  # DIGHOLO_ERROR_INVALIDDIMENSION
    L.digHoloDestroy(h)
