"""CUDA-graph replay of device-frame batches (digHoloB200SetGraphs): batches
on device-resident frames replay their captured forward and inverse
launches once the same launch arguments recur.  The replayed batches must
give exactly the results of direct launches, follow every change of the
frames, the configuration and the kernel choice, and fall back to direct
launches where the arguments are new.
"""
import ctypes as C

import numpy as np
import pytest

from digholo_b200 import api
from helpers import config_for, make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _coefs(lib, h, frames_dev, B):
    lib.digHoloSetBatchUint16(h, B, C.cast(C.c_void_p(frames_dev.data_ptr()), C.POINTER(C.c_ushort)), 0)
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    assert cp, lib.digHoloB200GetLastError(h)
    return np.ctypeslib.as_array(cp, shape=(b.value * m.value * pc.value * 2,)).copy()


@pytest.mark.parametrize("mode", [1, 0])
def test_graph_replay_equals_direct_launches(lib, mode):
    import torch
    B = 32
    hols = [make_case("batched_640x512_u16_2pol", B, seed=s) for s in (3, 4)]
    cfg = config_for(hols[0], mode)
    dev = [torch.from_numpy(np.ascontiguousarray(hh.frames).view(np.int16)).cuda() for hh in hols]
    hg = lib.digHoloCreate()
    hd = lib.digHoloCreate()
    for h in (hg, hd):
        api.configure(lib, h, cfg)
    assert lib.digHoloB200SetGraphs(hd, 0) == 0
    # two buffers in turn: each key runs directly, is captured, then replays
    for rnd in range(4):
        for i in (0, 1):
            g = _coefs(lib, hg, dev[i], B)
            d = _coefs(lib, hd, dev[i], B)
            np.testing.assert_array_equal(g, d)
    assert lib.digHoloB200GetGraphCount(hg) == 2
    assert lib.digHoloB200GetGraphCount(hd) == 0
    assert lib.digHoloB200GetForwardKernel(hg) == lib.digHoloB200GetForwardKernel(hd)
    assert lib.digHoloB200GetInverseKernel(hg) == lib.digHoloB200GetInverseKernel(hd)
    # a configuration change gives new launch arguments: results follow it
    for h in (hg, hd):
        lib.digHoloConfigSetTilt(h, 0, 0, float(cfg.tilt_deg[0][0]) + 0.01)
    for rnd in range(3):
        g = _coefs(lib, hg, dev[0], B)
        d = _coefs(lib, hd, dev[0], B)
        np.testing.assert_array_equal(g, d)
    assert lib.digHoloB200GetGraphCount(hg) == 3
    # an explicit kernel choice is part of the key as well
    for h in (hg, hd):
        assert lib.digHoloB200SetInverseKernel(h, 1) == 0
    for rnd in range(3):
        g = _coefs(lib, hg, dev[0], B)
        d = _coefs(lib, hd, dev[0], B)
        np.testing.assert_array_equal(g, d)
    assert lib.digHoloB200GetInverseKernel(hg) == 1
    assert lib.digHoloB200SetGraphs(hg, 0) == 0
    assert lib.digHoloB200GetGraphCount(hg) == 0
    for h in (hg, hd):
        lib.digHoloDestroy(h)


def test_default_stream_launches_directly(lib):
    """On the legacy default stream (digHoloB200SetStream with a null
    stream, as torch's default stream reports itself) nothing can be
    captured: the batches launch directly, with the same results."""
    import torch
    B = 16
    hol = make_case("batched_640x512_u16_2pol", B, seed=3)
    cfg = config_for(hol, 1)
    dev = torch.from_numpy(np.ascontiguousarray(hol.frames).view(np.int16)).cuda()
    hd = lib.digHoloCreate()
    hs = lib.digHoloCreate()
    for h in (hd, hs):
        api.configure(lib, h, cfg)
    ref = _coefs(lib, hs, dev, B)
    _coefs(lib, hd, dev, B)                       # first batch creates the handle's own stream
    assert lib.digHoloB200SetStream(hd, None) == 0
    for _ in range(3):
        np.testing.assert_array_equal(_coefs(lib, hd, dev, B), ref)
    assert lib.digHoloB200GetGraphCount(hd) == 0
    for h in (hd, hs):
        lib.digHoloDestroy(h)
