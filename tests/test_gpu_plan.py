"""The kernel planner: FFTW plan modes above ESTIMATE (digHoloConfigSetFFTWPlanMode,
digHolo.h:1808) time every forward x inverse kernel pair on the first batch
of a shape and use the fastest afterwards; the plans are kept like FFTW's
wisdom (digHoloFFTWWisdomForget / digHoloFFTWWisdomFilename,
digHolo.h:1825-1835).

Checked: the first batch of a shape records a plan, and it and the batches
after it (processed with the planned kernels) match the oracle at the
tolerances of test_gpu_parity.py; a second handle with the same shape uses
the plan without timing again; forgetting the plans and naming the wisdom
file again restores them from the file, again without timing.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
from digholo_b200 import api
from helpers import config_for, make_case, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _plan(lib, h):
    f, i, ms = C.c_int(-1), C.c_int(-1), C.c_float(0)
    found = lib.digHoloB200GetKernelPlan(h, C.byref(f), C.byref(i), C.byref(ms))
    return found, f.value, i.value, ms.value


def _check(g, o, split_bf16):
    dR = np.abs(g["R"].astype(np.int32) - o["R"])
    dI = np.abs(g["I"].astype(np.int32) - o["I"])
    assert max(int(dR.max()), int(dI.max())) <= 2
    assert rel_l2(g["field"], o["field"]) <= 5e-5
    assert rel_l2(g["coefs"], o["coefs"]) <= (1e-4 if split_bf16 else 5e-5)


@pytest.mark.parametrize("workload,frames,mode", [("batched_640x512_u16_2pol", 64, 1),
                                                  ("batched_640x512_u16_2pol", 64, 0),
                                                  ("plain_320x256_f32_1pol", 64, 1)])
def test_planned_batches_match_oracle(lib, tmp_path, workload, frames, mode):
    wisdom = str(tmp_path / "plans.txt")
    assert lib.digHoloFFTWWisdomFilename(wisdom.encode()) == 0
    assert lib.digHoloFFTWWisdomForget() == 0
    hol = make_case(workload, frames)
    cfg = config_for(hol, mode)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    assert lib.digHoloConfigSetFFTWPlanMode(h, 1) == 0
    runs0 = lib.digHoloB200GetKernelPlanRuns()
    g = api.run_batch(lib, h, hol.frames)
    assert lib.digHoloB200GetKernelPlanRuns() == runs0 + 1
    found, f, i, ms = _plan(lib, h)
    print("%s mode %d: planned forward %d inverse %d, %.3f ms per batch" % (workload, mode, f, i, ms))
    assert found == 1 and f in (1, 2, 3, 4, 5) and i in (0, 1, 2, 3) and ms > 0
    _check(g, o, lib.digHoloB200GetOverlapKernel(h) == 2)
    for _ in range(2):   # later batches run the planned pair
        g = api.run_batch(lib, h, hol.frames)
        _check(g, o, lib.digHoloB200GetOverlapKernel(h) == 2)
    assert lib.digHoloB200GetKernelPlanRuns() == runs0 + 1
    # another handle of the same shape: no second timing
    h2 = lib.digHoloCreate()
    api.configure(lib, h2, cfg)
    lib.digHoloConfigSetFFTWPlanMode(h2, 1)
    api.run_batch(lib, h2, hol.frames, want_fields=False)
    assert lib.digHoloB200GetKernelPlanRuns() == runs0 + 1
    # forgotten, then restored from the wisdom file
    assert lib.digHoloFFTWWisdomForget() == 0
    assert _plan(lib, h2)[0] == 0
    assert lib.digHoloFFTWWisdomFilename(wisdom.encode()) == 0
    assert _plan(lib, h2)[:3] == (1, f, i)
    api.run_batch(lib, h2, hol.frames, want_fields=False)
    assert lib.digHoloB200GetKernelPlanRuns() == runs0 + 1
    lib.digHoloDestroy(h)
    lib.digHoloDestroy(h2)
    assert open(wisdom).readline().strip() == "digholo_b200 kernel plans v1"


def test_estimate_mode_does_not_plan(lib):
    hol = make_case("batched_640x512_u16_2pol", 16)
    cfg = config_for(hol, 1)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    assert lib.digHoloConfigSetFFTWPlanMode(h, 0) == 0
    runs0 = lib.digHoloB200GetKernelPlanRuns()
    api.run_batch(lib, h, hol.frames, want_fields=False)
    assert lib.digHoloB200GetKernelPlanRuns() == runs0
    lib.digHoloDestroy(h)
