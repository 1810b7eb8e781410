"""The oracle (FP64 restatement) pinned against the reference.

* against the committed golden fixtures (outputs of the unmodified reference,
  tests/golden/make_golden.py), which need no reference build;
* against the live reference build (oracle/_ref) where it exists.

Tolerances: int16 fields within 2 LSB and field relative L2 <= 5e-5; coefficient
relative L2 <= 2e-5 (for 16-row fields after removing the scale the
reference omits, digHolo.cpp:2318-2331); field scales relative <= 1e-5.
"""
import glob
import json
import os

import numpy as np
import pytest

import digholo_oracle as O
import ref_lib
from helpers import config_for, make_case, rel_l2

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _check(o, cfg, coefs, R, I, scale, x, y):
    np.testing.assert_array_equal(x, o["x"])
    np.testing.assert_array_equal(y, o["y"])
    dR = np.abs(R.astype(int) - o["R"])
    dI = np.abs(I.astype(int) - o["I"])
    assert max(dR.max(), dI.max()) <= 2
    assert np.max(np.abs(scale.T - o["scale"]) / o["scale"]) <= 1e-5
    # one 14-bit reference-wave entry rounded the other way shifts a whole row
    # or column by 1 LSB, so compare the fields, not the count of differing values
    f = (R + 1j * I.astype(np.float64)) / scale.T[:, :, None, None]
    fo = (o["R"] + 1j * o["I"].astype(np.float64)) / o["scale"][:, :, None, None]
    assert rel_l2(f, fo) <= 5e-5
    co = o["coefs"]
    if o["h"] == 16 and cfg.resolution_mode == 1:
        co = O.reference_unscaled_16(co, cfg, o)
    assert rel_l2(coefs, co) <= 2e-5


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path):
    d = np.load(path)
    meta = json.loads(str(d["meta"]))
    hol = make_case(meta["workload"], meta["frames"])
    cfg = config_for(hol, meta["mode"])
    o = O.process_batch(hol.frames, cfg, quantised=True)
    _check(o, cfg, d["coefs"], d["R"], d["I"], d["scale"], d["x"], d["y"])


def test_golden_fixtures_present():
    assert len(GOLDEN) == 4


@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_matches_live_reference(mode):
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    hol = make_case("plain_320x256_f32_1pol", 4)
    cfg = config_for(hol, mode)
    L = ref_lib.load()
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    r = ref_lib.run_batch(L, h, hol.frames)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    _check(o, cfg, r["coefs"], r["R"], r["I"], r["scale"], r["x"], r["y"])


def test_exact_and_quantised_flavours_agree():
    hol = make_case("plain_320x256_f32_1pol", 2)
    cfg = config_for(hol, 0)
    q = O.process_batch(hol.frames, cfg, quantised=True)
    e = O.process_batch(hol.frames, cfg, quantised=False)
    # the quantisation of the reference (int16 field, 14-bit wave, int16 modes) costs ~5e-5
    assert rel_l2(q["field"], e["field"]) < 2e-4
    assert rel_l2(q["coefs"], e["coefs"]) < 1e-4


def test_metrics_on_unitary_batch():
    # a batch whose coefficient matrix is unitary has IL = MDL = 0 dB on both paths
    rng = np.random.default_rng(7)
    z = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    q, _ = np.linalg.qr(z)
    m = O.power_meter(q.T.reshape(6, 1, 6))
    assert abs(m["il_db"]) < 1e-9 and abs(m["mdl_db"]) < 1e-9
    assert abs(m["il_frob_db"]) < 1e-9


def check_fourier(o, f, cfg, plane_tol=1e-6):
    """Plane-0 outputs (Fourier plane, its statistics and batch sum) against
    the oracle: plane relative L2 <= plane_tol, power / CoM / Aeff / scale
    relative <= 1e-4 (FP32 sums over the plane), the maximum's index equal,
    batch-sum plane relative L2 <= 1e-5 over the analysed pixels."""
    P = cfg.pol_count
    planes = o["fourier"]
    assert rel_l2(f["plane"], planes) <= plane_tol
    assert f["width"] == o["W"]
    s = f["summary"]
    for pol in range(P):
        st = o["fft_stats"][pol]
        for k, name in ((0, "power"), (1, "comx"), (2, "comy"), (5, "aeff"), (6, "comywrap"), (3, "scale")):
            got = s[k, pol].astype(np.float64)
            ref = st[name]
            assert np.all(np.abs(got - ref) <= 1e-4 * np.abs(ref) + 1e-30), (name, got, ref)
        np.testing.assert_array_equal(s[4, pol].view(np.int32), st["maxidx"])
        bs = f["batchsum"][pol]
        assert rel_l2(bs, st["batchsum"]) <= 1e-5


@pytest.mark.parametrize("workload", ["plain_320x256_f32_1pol", "batched_640x512_u16_2pol"])
def test_fourier_analysis_matches_live_reference(workload):
    """The FFT-stage analysis of the oracle against the reference's own
    digHoloGetFourierPlaneFull and digHoloBatchGetSummary(plane 0)."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    from digholo_b200 import api
    hol = make_case(workload, 4)
    cfg = config_for(hol, 1)
    L = ref_lib.load()
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    ref_lib.run_batch(L, h, hol.frames)
    f = api.read_fourier(L, h)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    check_fourier(o, f, cfg)


@pytest.mark.parametrize("res_mode,avg_mode", [(1, 0), (1, 1), (0, 0)])
def test_frame_averaging_matches_live_reference(res_mode, avg_mode):
    """Frame averaging (digHoloSetBatchAvg, 3 frames per batch item): the
    oracle's phase-aligned window average against the reference build."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    import ctypes as C
    from digholo_b200 import api
    hol = make_case("plain_320x256_f32_1pol", 6)
    cfg = config_for(hol, res_mode)
    cfg.avg_count, cfg.avg_mode = 3, avg_mode
    L = ref_lib.load()
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    frames = np.ascontiguousarray(hol.frames.astype(np.float32))
    api.set_batch_avg(L, h, frames, 3, avg_mode)
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    r = api.read_outputs(L, h, 2, cp, m.value, p.value, True)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    assert o["R"].shape[0] == 2
    _check(o, cfg, r["coefs"], r["R"], r["I"], r["scale"], r["x"], r["y"])


@pytest.mark.parametrize("avg", [1, 3])
def test_batch_calibration_matches_live_reference(avg):
    """Batch calibration (digHoloConfigSetBatchCalibration: one complex
    factor per polarisation and batch item, applied to the Fourier windows),
    without and with frame averaging: the oracle against the reference build."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    import ctypes as C
    from digholo_b200 import api
    hol = make_case("batched_640x512_u16_2pol", 4 * avg)
    cfg = config_for(hol, 1)
    rng = np.random.default_rng(11)
    cfg.batch_cal = (rng.uniform(0.5, 2.0, (2, 3)) * np.exp(1j * rng.uniform(-np.pi, np.pi, (2, 3))))
    cfg.avg_count, cfg.avg_mode = avg, 0
    L = ref_lib.load()
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    api.set_batch_avg(L, h, np.ascontiguousarray(hol.frames), avg, 0)
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    r = api.read_outputs(L, h, 4, cp, m.value, p.value, True)
    o = O.process_batch(hol.frames, cfg, quantised=True)
    _check(o, cfg, r["coefs"], r["R"], r["I"], r["scale"], r["x"], r["y"])


@pytest.mark.parametrize("basis", ["lg", "custom"])
def test_basis_transform_matches_live_reference(basis):
    """Coefficients in the Laguerre-Gaussian basis and in a custom basis
    (digHoloConfigSetBasisTypeLG / Custom, 45 HG modes onto 30 custom modes):
    the oracle's transform of its HG coefficients against the reference
    build's returned coefficients (full resolution: no unscaled 16-row case)."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    import ctypes as C
    from digholo_b200 import api
    hol = make_case("plain_320x256_f32_1pol", 8)
    cfg = config_for(hol, 0)
    if basis == "lg":
        cfg.basis_type = 1
    else:
        rng = np.random.default_rng(5)
        cfg.basis_type = 2
        cfg.basis_custom = (rng.normal(size=(50, 30)) + 1j * rng.normal(size=(50, 30))).astype(np.complex64)
    L = ref_lib.load()
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    frames = np.ascontiguousarray(hol.frames.astype(np.float32))
    api.set_batch(L, h, frames)
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    o = O.process_batch(hol.frames, cfg, quantised=True)
    co = o["coefs_out"]
    assert m.value == co.shape[2] and b.value == co.shape[0]
    r = np.ctypeslib.as_array(cp, shape=(b.value * m.value * p.value * 2,)).copy().view(np.complex64).reshape(co.shape)
    assert rel_l2(r, co) <= 2e-5
    if basis == "lg":
        # the LG transform is unitary: the power per frame is unchanged
        np.testing.assert_allclose(np.sum(np.abs(co) ** 2, axis=(1, 2)), np.sum(np.abs(o["coefs"]) ** 2, axis=(1, 2)),
                                   rtol=1e-6)


def test_lg_transform_is_block_unitary():
    """The oracle's HG -> LG matrix: block-diagonal by mode group, each block
    unitary (to complex64 rounding), and the l = +-g modes of group g carry
    the binomial weights sqrt(C(g, k) / 2^g) in magnitude."""
    import math
    G = 8
    T = O.lg_transform(G)
    M = G * (G + 1) // 2
    assert T.shape == (M, M)
    base = 0
    for g in range(G):
        blk = T[base:base + g + 1, base:base + g + 1]
        np.testing.assert_allclose(blk.conj().T @ blk, np.eye(g + 1), atol=1e-6)
        off = np.abs(T[base:base + g + 1, :]).sum() - np.abs(blk).sum()
        assert off == 0.0
        mag = np.abs(blk[:, 0])   # LG l = g: weights over the HG modes of the group
        want = np.array([math.sqrt(math.comb(g, k) / 2.0 ** g) for k in range(g + 1)])
        np.testing.assert_allclose(np.sort(mag), np.sort(want), atol=1e-6)
        base += g + 1


def test_snap_estimate_matches_live_reference():
    """The oracle's AutoAlign parameter estimate (auto_align_snap, restating
    digHoloAutoAlignSnap digHolo.cpp:11517-11970 and digHoloAutoFocus
    digHolo.cpp:11181-11499) against the reference's ESTIMATE mode from a
    cold start (beam centres and tilts 0, waist 400 um), without the
    window-radius rule, low-resolution fields, single-threaded reference.
    Tilts equal, beam centres within 1 nm, waist within 1e-4 relative,
    first polarisation's defocus within 1e-3 (the second's is not compared:
    the reference's focus search reads unwritten memory for it past its
    22nd trial, digHolo.cpp:11434)."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    import ctypes as C
    from digholo_b200 import api, synth
    B = 16
    kw = dict(synth.WORKLOADS["snap_640x512_f32_2pol"])
    kw.update(frame_count=B, coefs=synth.transfer_coefs(B, 2, kw["max_mg"], 1004))
    hol = synth.generate(**kw)
    cfg = config_for(hol, 1)
    for p in range(2):
        cfg.beam_centre[p] = [O.F32(0), O.F32(0)]
        cfg.tilt_deg[p] = [O.F32(0), O.F32(0)]
        cfg.waist[p] = O.F32(400e-6)
    fr = np.ascontiguousarray(hol.frames.astype(np.float32))
    L = ref_lib.load()
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    L.digHoloConfigSetThreadCount(h, 1)
    L.digHoloSetBatch(h, B, fr.ctypes.data_as(C.POINTER(C.c_float)))
    L.digHoloConfigSetAutoAlignMode(h, 2)
    L.digHoloConfigSetAutoAlignFourierWindowRadius(h, 0)
    L.digHoloAutoAlign(h)
    c, steps, info = O.auto_align_snap(fr, cfg, align_radius=0)
    for p in range(2):
        for ax in range(2):
            assert L.digHoloConfigGetTilt(h, ax, p) == pytest.approx(float(c.tilt_deg[p][ax]), abs=1e-6)
            assert abs(L.digHoloConfigGetBeamCentre(h, ax, p) - float(c.beam_centre[p][ax])) <= 1e-9
    assert abs(L.digHoloConfigGetBasisWaist(h, 0) - float(c.waist[0])) <= 1e-4 * float(c.waist[0])
    assert abs(L.digHoloConfigGetDefocus(h, 0) - float(c.defocus[0])) <= 1e-3


def _ref_simulate(L, frames, W, H, P, G, levels, fill, coefs=None, waist=None, tiltx=None):
    """The reference build's digHoloFrameSimulatorCreate (digHolo.cpp:16755)."""
    import ctypes as C
    Wc, Hc, psc, Pc, Gc, lv, wc = C.c_int(W), C.c_int(H), C.c_float(20e-6), C.c_int(P), C.c_int(G), C.c_int(levels), C.c_int(0)
    nul = lambda: C.POINTER(C.c_float)()
    keep = []

    def arr(v):
        if v is None:
            return C.pointer(nul())
        a = np.ascontiguousarray(np.asarray(v, dtype=np.complex64).view(np.float32) if np.iscomplexobj(v)
                                 else np.asarray(v, dtype=np.float32))
        keep.append(a)
        return C.pointer(a.ctypes.data_as(C.POINTER(C.c_float)))
    p16 = C.POINTER(C.c_ushort)()
    out = L.digHoloFrameSimulatorCreate(frames, C.byref(Wc), C.byref(Hc), C.byref(psc), C.byref(Pc), arr(tiltx),
                                        arr(None), arr(None), arr(None), arr(None), arr(None), arr(None), C.byref(Gc),
                                        arr(waist), arr(coefs), arr(None), arr(None), C.byref(lv), fill, arr(None),
                                        C.byref(wc), 0, 0, C.byref(p16), None)
    n = frames * Hc.value * Wc.value
    f32 = np.ctypeslib.as_array(out, shape=(n,)).copy().reshape(frames, Hc.value, Wc.value)
    L.digHoloFrameSimulatorDestroy(out)
    return f32, Gc.value


@pytest.mark.parametrize("case", [(6, 128, 64, 2, 3, 16384, 0, False), (10, 160, 96, 2, 0, 16384, 1, False),
                                  (5, 192, 128, 2, 5, 4096, 1, True), (4, 128, 128, 1, 6, 4096, 0, True)])
def test_frame_simulator_matches_live_reference(case):
    """The frame simulator restatement against the reference build: the
    same group count, and frames equal except at no more than 1e-4 of the
    pixels, by one camera level (float rounding of the reference's scalar
    tables)."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    fr, W, H, P, G, levels, fill, dense = case
    coefs = waist = tiltx = None
    if dense:
        rng = np.random.default_rng(3 + fr)
        M = G * (G + 1) // 2
        coefs = (rng.standard_normal((fr, P, M)) + 1j * rng.standard_normal((fr, P, M))).astype(np.complex64)
        coefs[:, :, 3] = 0
        waist, tiltx = [300e-6, 250e-6][:P], [1.5, -1.2][:P]
    r32, Gr = _ref_simulate(ref_lib.load(), fr, W, H, P, G, levels, fill, coefs, waist, tiltx)
    o32, o16, prm = O.frame_simulator(fr, W, H, 20e-6, P, group_count=G, levels=levels, fill_factor=fill,
                                      beam_coefs=coefs, beam_waist=waist, ref_tilt_x=tiltx)
    assert prm["G"] == Gr
    d = np.abs(r32 - o32)
    assert d.max() <= 1 and float((d > 0).mean()) <= 1e-4


@pytest.mark.parametrize("workload,mode,kind,count,window", [
    ("plain_320x256_f32_1pol", 1, "intensity", 1, None), ("plain_320x256_f32_1pol", 0, "field", 3, None),
    ("batched_640x512_u16_2pol", 1, "field", 1, None), ("batched_640x512_u16_2pol", 0, "intensity", 2, None),
    ("batched_640x512_u16_2pol", 0, "intensity", 1, 256), ("largefield_2048_u16_2pol", 0, "intensity", 1, None)])
def test_ref_calibration_matches_live_reference(workload, mode, kind, count, window):
    """Reference-wave calibration (digHoloConfigSetRefCalibrationIntensity /
    Field): the oracle's reconstructed calibration planes against the
    reference's digHoloConfigGetRefCalibrationFields (relative L2 <= 1e-6),
    and the calibrated batch's fields and coefficients against the
    reference's (the usual bounds).  The calibration changes the
    coefficients by 0.8-9 % here, well above the comparison's bounds.  The
    reference runs in a child process (helpers.reference_calibrated)."""
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    from helpers import ref_calibration, reference_calibrated
    frames = 1 if workload.startswith("largefield") else 2
    hol = make_case(workload, frames)
    cfg = config_for(hol, mode)
    if window:
        cfg.fft_window = (window, window)
    cfg.ref_cal = (O.ref_cal_store(intensity=ref_calibration(cfg, kind, count)) if kind == "intensity"
                   else O.ref_cal_store(field=ref_calibration(cfg, kind, count)))
    r = reference_calibrated(workload, frames, mode, kind, count, window)
    op = O.ref_cal_planes(cfg)
    assert r["planes"].shape == op.shape
    assert rel_l2(op, r["planes"]) <= 1e-6
    o = O.process_batch(hol.frames, cfg, quantised=True)
    _check(o, cfg, r["coefs"], r["R"], r["I"], r["scale"], r["x"], r["y"])
    plain = config_for(hol, mode)
    if window:
        plain.fft_window = (window, window)
    assert rel_l2(O.process_batch(hol.frames, plain, quantised=True)["coefs"], o["coefs"]) > 3e-3
