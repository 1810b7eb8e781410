"""Parity at the benchmarked size: 1024 frames of 640x512 uint16, two
polarisations, 128x128 FFT windows, 120 modes (maxMG 15) -- the batch the
throughput figure is measured on -- and 3072 frames of 320x256 float32.

At these sizes every block of the persistent forward kernels runs many
units: the tensor-core forward (k_forward_i8) launches min(SMs, frames x
pol) blocks and each walks frames frame0, frame0 + grid/P, ..., so with
1024 dual-polarisation frames each block runs ceil(1024 / (grid/2)) >= 4
units, wrapping its TMA stage ring (4 stages), its two tensor-memory
accumulator sets and their empty/full hand-offs many times.  The TMA-fed
float kernel (k_forward_tma) walks units with a stride of its grid (at most
5 blocks per SM fit its shared memory and registers with 64x64 windows), so
3072 single-polarisation frames give each block at least 4 units as well.

Every frame's int16 fields, field scales and coefficients are compared with
the oracle (the FP64 restatement, quantised like the reference) at the
tolerances of test_gpu_parity.py: int16 fields within 2 LSB, field relative
L2 <= 5e-5, scales <= 1e-5 relative, coefficients relative L2 <= 5e-5 (FP32
overlap) or <= 1e-4 (split-BF16 tensor-core overlap); a strided subset of
the frames is compared with the reference build as well.
"""
import ctypes as C

import numpy as np
import pytest

import digholo_oracle as O
import ref_lib
from digholo_b200 import api
from helpers import config_for, make_case, rel_l2

pytestmark = pytest.mark.gpu

FRAMES = 1024
FLOAT_FRAMES = 3072
STRIDE = 37          # every 37th frame also goes through the reference build


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


@pytest.fixture(scope="module")
def hol():
    return make_case("batched_640x512_u16_2pol", FRAMES, seed=2002)


_ORACLE = {}


def _oracle(hol, mode):
    if mode not in _ORACLE:
        _ORACLE[mode] = O.process_batch(hol.frames, config_for(hol, mode), quantised=True)
    return _ORACLE[mode]


def _sm_count():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count


def _check(g, o, split_bf16):
    assert g["R"].shape == o["R"].shape
    dR = np.abs(g["R"].astype(np.int32) - o["R"])
    dI = np.abs(g["I"].astype(np.int32) - o["I"])
    assert max(int(dR.max()), int(dI.max())) <= 2
    scale_rel = np.max(np.abs(g["scale"].T - o["scale"]) / o["scale"])
    assert scale_rel <= 1e-5, scale_rel
    # every frame on its own, not only the batch as a whole
    B = g["field"].shape[0]
    fe = [rel_l2(g["field"][f], o["field"][f]) for f in range(B)]
    assert max(fe) <= 5e-5, (int(np.argmax(fe)), max(fe))
    tol = 1e-4 if split_bf16 else 5e-5
    ce = [rel_l2(g["coefs"][f], o["coefs"][f]) for f in range(B)]
    assert max(ce) <= tol, (int(np.argmax(ce)), max(ce))


def _run(lib, h, frames):
    return api.run_batch(lib, h, frames)


@pytest.mark.parametrize("mode,inverse", [(1, 0), (1, 3), (0, 0)])
def test_headline_batch_every_frame(lib, hol, mode, inverse):
    """Host frames through digHoloSetBatchUint16 + digHoloProcessBatch."""
    P = hol.pol_count
    grid = min(_sm_count(), FRAMES * P) // P * P
    units_per_block = -(-FRAMES // (grid // P))
    assert units_per_block >= 4, units_per_block
    cfg = config_for(hol, mode)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    assert lib.digHoloB200SetInverseKernel(h, inverse) == 0
    g = _run(lib, h, hol.frames)
    fwd, inv = lib.digHoloB200GetForwardKernel(h), lib.digHoloB200GetInverseKernel(h)
    ovl = lib.digHoloB200GetOverlapKernel(h)
    lib.digHoloDestroy(h)
    assert fwd == 4                                  # the tensor-core forward ran
    if inverse == 3:
        assert inv == 5                              # forward and inverse fused in one launch
    else:
        assert inv == (2 if mode == 1 else 3)
    _check(g, _oracle(hol, mode), split_bf16=(ovl == 2))


@pytest.mark.parametrize("mode", [1, 0])
def test_headline_batch_vs_reference_build(lib, hol, mode):
    """A strided subset of the frames through the reference build: frames
    are independent, so the subset's results equal those rows of the full
    batch's."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    cfg = config_for(hol, mode)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    g = _run(lib, h, hol.frames)
    lib.digHoloDestroy(h)
    sub = np.ascontiguousarray(hol.frames[::STRIDE])
    L = ref_lib.load()
    hr = L.digHoloCreate()
    ref_lib.configure(L, hr, cfg)
    r = ref_lib.run_batch(L, hr, sub)
    gf = g["field"][::STRIDE]
    assert rel_l2(gf, r["field"]) <= 5e-5
    o = _oracle(hol, mode)
    gc = g["coefs"][::STRIDE].astype(np.complex128)
    if o["h"] == 16 and mode == 1:
        # the reference leaves 16-row fields unscaled (digHolo.cpp:2318-2331); this build scales them
        osub = dict(o)
        osub["scale"] = o["scale"][::STRIDE]
        gc = O.reference_unscaled_16(gc, cfg, osub)
    tol = 1e-4 if mode == 0 else 5e-5
    assert rel_l2(gc, r["coefs"]) <= tol


@pytest.mark.parametrize("mode", [1, 0])
def test_headline_graph_replay_every_frame(lib, hol, mode):
    """Device-resident frames with CUDA-graph replay: two frame buffers in
    turn, three rounds (each buffer runs directly, is captured, then
    replays); every result against the oracle."""
    import torch
    cfg = config_for(hol, mode)
    half = FRAMES // 2
    # two buffers, each a full 1024-frame batch: the first half of the batch
    # rolled to the front of the second buffer
    order = [np.arange(FRAMES), np.roll(np.arange(FRAMES), half)]
    dev = [torch.from_numpy(np.ascontiguousarray(hol.frames[idx]).view(np.int16)).cuda() for idx in order]
    o = _oracle(hol, mode)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    for rnd in range(3):
        for i in (0, 1):
            fp = C.cast(C.c_void_p(dev[i].data_ptr()), C.POINTER(C.c_ushort))
            assert lib.digHoloSetBatchUint16(h, FRAMES, fp, 0) == 0
            b, m, pc = C.c_int(), C.c_int(), C.c_int()
            cp = lib.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
            assert cp, lib.digHoloB200GetLastError(h)
            g = api.read_outputs(lib, h, FRAMES, cp, m.value, pc.value, want_fields=True)
            oi = {k: (o[k][order[i]] if k in ("R", "I", "field", "coefs") else o[k]) for k in ("R", "I", "field", "coefs")}
            oi["scale"] = o["scale"][order[i]]
            _check(g, oi, split_bf16=(lib.digHoloB200GetOverlapKernel(h) == 2))
    assert lib.digHoloB200GetGraphCount(h) == 2
    lib.digHoloDestroy(h)


@pytest.mark.parametrize("mode", [1, 0])
def test_float_frames_persistent_loop(lib, mode):
    """3072 frames of 320x256 float32 (one polarisation, 64x64 window):
    k_forward_tma runs at least 4 units per block."""
    hol = make_case("plain_320x256_f32_1pol", FLOAT_FRAMES, seed=2003)
    assert FLOAT_FRAMES >= 4 * 5 * _sm_count()
    cfg = config_for(hol, mode)
    h = lib.digHoloCreate()
    api.configure(lib, h, cfg)
    g = _run(lib, h, hol.frames)
    fwd = lib.digHoloB200GetForwardKernel(h)
    ovl = lib.digHoloB200GetOverlapKernel(h)
    lib.digHoloDestroy(h)
    assert fwd == 3
    o = O.process_batch(hol.frames, cfg, quantised=True)
    _check(g, o, split_bf16=(ovl == 2))
