"""Adjoint (gradient) of the batch path and the gradient-driven AutoAlign.

Workload: frames exciting the columns of a Haar-random transfer matrix with
per-mode loss (synth.transfer_coefs), dual polarisation, 120 modes, the
alignment perturbed from the true one (beam centre +30/-20 um, tilt +-2 %,
waist +10 %).

* digHoloB200AutoAlignGradient against central finite differences of the
  same objective IL = 10 log10(sum |c|^2): steps of 5 % of the reference's
  AutoAlign step sizes (tilt 0.1 x window radius, centre and waist 0.1 x
  waist, defocus 0.4), each component within 5 % of the gradient norm and
  cosine similarity >= 0.99;
* a torch.autograd.Function around the library runs torch.autograd.gradcheck
  in step-normalised coordinates (the test harness is the only torch user);
* digHoloB200AutoAlignAdjoint reaches the plain search's (digHoloAutoAlign,
  TWEAK) goal metric within 0.01 dB: IL for goal IL (the MDL at the point
  each search reaches is printed; it is not what either search maximises),
  MDL for goal MDL (its IL is printed: the MDL pass trades IL for MDL in
  both searches) -- both metrics: higher is better; MDL in dB is
  s_min^2 / s_max^2 <= 1.  In IFFT resolution mode 1 the reconstructed
  field is 16 pixels across: a waist below a pixel leaves the sampled basis
  unnormalised and the IL objective grows without bound there (the plain
  search runs into the waist limit), so that comparison holds the waist.
"""
import ctypes as C
import time

import numpy as np
import pytest

from digholo_b200 import api, synth
from helpers import config_for

pytestmark = pytest.mark.gpu

KINDS = ["tiltX", "tiltY", "defocus", "beamCentreX", "beamCentreY", "waist"]


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _case(frames, seed=77):
    kw = dict(synth.WORKLOADS["align_640x512_f32_2pol"])
    kw["frame_count"] = frames
    kw["coefs"] = synth.transfer_coefs(frames, 2, kw["max_mg"], seed)
    return synth.generate(**kw)


def _perturbed(hol, mode):
    cfg = config_for(hol, mode)
    cfg.beam_centre = [[bc[0] + 30e-6, bc[1] - 20e-6] for bc in cfg.beam_centre]
    cfg.tilt_deg = [[t[0] * 1.02, t[1] * 0.98] for t in cfg.tilt_deg]
    cfg.waist = [w * 1.1 for w in cfg.waist]
    return cfg


def _handle(L, cfg, frames):
    h = L.digHoloCreate()
    api.configure(L, h, cfg)
    fr = np.ascontiguousarray(frames)
    api.set_batch(L, h, fr)
    b, m, p = C.c_int(), C.c_int(), C.c_int()
    L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
    return h, fr


def _get(L, h, pol, kind):
    if kind == "tiltX": return L.digHoloConfigGetTilt(h, 0, pol)
    if kind == "tiltY": return L.digHoloConfigGetTilt(h, 1, pol)
    if kind == "defocus": return L.digHoloConfigGetDefocus(h, pol)
    if kind == "beamCentreX": return L.digHoloConfigGetBeamCentre(h, 0, pol)
    if kind == "beamCentreY": return L.digHoloConfigGetBeamCentre(h, 1, pol)
    return L.digHoloConfigGetBasisWaist(h, pol)


def _set(L, h, pol, kind, v):
    if kind == "tiltX": return L.digHoloConfigSetTilt(h, 0, pol, v)
    if kind == "tiltY": return L.digHoloConfigSetTilt(h, 1, pol, v)
    if kind == "defocus": return L.digHoloConfigSetDefocus(h, pol, v)
    if kind == "beamCentreX": return L.digHoloConfigSetBeamCentre(h, 0, pol, v)
    if kind == "beamCentreY": return L.digHoloConfigSetBeamCentre(h, 1, pol, v)
    return L.digHoloConfigSetBasisWaist(h, pol, v)   # sets every polarisation's waist


def _grad(L, h):
    g = (C.c_float * 12)()
    il = C.c_float()
    assert L.digHoloB200AutoAlignGradient(h, g, C.byref(il)) == 0, L.digHoloB200GetLastError(h)
    return np.array(g[:], dtype=np.float64).reshape(2, 6), float(il.value)


def _grad_metric(L, h, metric):
    g = (C.c_float * 12)()
    v = C.c_float()
    assert L.digHoloB200AutoAlignGradientMetric(h, metric, g, C.byref(v)) == 0, L.digHoloB200GetLastError(h)
    return np.array(g[:], dtype=np.float64).reshape(2, 6), float(v.value)


def _steps(L, h, cfg):
    radius = L.digHoloConfigGetFourierWindowRadius(h)
    w = cfg.waist[0]
    return {"tiltX": 0.1 * radius, "tiltY": 0.1 * radius, "defocus": 0.4,
            "beamCentreX": 0.1 * w, "beamCentreY": 0.1 * w, "waist": 0.1 * w}


# maxMG 15 and 20 run the register-tiled gradient kernel (16- and 32-mode
# tiles).  Beyond 32 groups (the generic kernel) the basis spans these
# 128-pixel fields: IL no longer depends on the alignment and finite
# differences are noise.
@pytest.mark.parametrize("mode,max_mg", [(0, None), (1, None), (0, 20)])
def test_gradient_vs_finite_differences(lib, mode, max_mg):
    hol = _case(32)
    cfg = _perturbed(hol, mode)
    if max_mg:
        cfg.max_mg = max_mg
    h, _ = _handle(lib, cfg, hol.frames)
    assert lib.digHoloB200FreezeWindow(h, 1) == 0   # windows frozen, as the gradient assumes
    g, il0 = _grad(lib, h)
    steps = _steps(lib, h, cfg)
    # the waist setter moves both polarisations: compare with the summed gradient
    entries = [(pol, k) for pol in (0, 1) for k in KINDS[:5]] + [(None, "waist")]
    ga, gf = [], []
    for pol, kind in entries:
        p0 = 0 if pol is None else pol
        base = _get(lib, h, p0, kind)
        d = 0.05 * steps[kind]
        vals = []
        for sgn in (1, -1):
            _set(lib, h, p0, kind, base + sgn * d)
            vals.append(_grad(lib, h)[1])
        _set(lib, h, p0, kind, base)
        gf.append((vals[0] - vals[1]) / (2 * d) * steps[kind])
        ga.append((g[0, 5] + g[1, 5] if pol is None else g[pol, KINDS.index(kind)]) * steps[kind])
    lib.digHoloDestroy(h)
    ga, gf = np.array(ga), np.array(gf)
    print("mode %d maxMG %s IL %.4f dB; gradient x step (dB):" % (mode, max_mg or hol.max_mg, il0))
    for (pol, kind), a, f in zip(entries, ga, gf):
        print("  pol %s %-12s adjoint % .5f  finite difference % .5f" % (pol, kind, a, f))
    norm = np.linalg.norm(gf)
    cos = float(ga @ gf / (np.linalg.norm(ga) * norm))
    assert cos >= 0.99, cos
    assert np.max(np.abs(ga - gf)) <= 0.05 * norm, (ga, gf)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("independent", [0, 1])
def test_mdl_gradient_vs_finite_differences(lib, mode, independent):
    """MDL = 10 log10(lambda_min / lambda_max) of the batch Gram matrix (both
    polarisations together, or the extremes over the two polarisations'
    blocks): the adjoint gradient through d lambda = u^H dG u against central
    differences of the same MDL, windows frozen; cosine >= 0.99, each
    component within 5 % of the norm."""
    hol = _case(32)
    cfg = _perturbed(hol, mode)
    h, _ = _handle(lib, cfg, hol.frames)
    lib.digHoloConfigSetAutoAlignPolIndependence(h, independent)
    assert lib.digHoloB200FreezeWindow(h, 1) == 0
    g, m0 = _grad_metric(lib, h, 1)
    steps = _steps(lib, h, cfg)
    entries = [(pol, k) for pol in (0, 1) for k in KINDS[:5]] + [(None, "waist")]
    ga, gf = [], []
    for pol, kind in entries:
        p0 = 0 if pol is None else pol
        base = _get(lib, h, p0, kind)
        d = 0.05 * steps[kind]
        vals = []
        for sgn in (1, -1):
            _set(lib, h, p0, kind, base + sgn * d)
            vals.append(_grad_metric(lib, h, 1)[1])
        _set(lib, h, p0, kind, base)
        gf.append((vals[0] - vals[1]) / (2 * d) * steps[kind])
        ga.append((g[0, 5] + g[1, 5] if pol is None else g[pol, KINDS.index(kind)]) * steps[kind])
    lib.digHoloDestroy(h)
    ga, gf = np.array(ga), np.array(gf)
    print("mode %d independent %d MDL %.4f dB; gradient x step (dB):" % (mode, independent, m0))
    for (pol, kind), a, f in zip(entries, ga, gf):
        print("  pol %s %-12s adjoint % .5f  finite difference % .5f" % (pol, kind, a, f))
    assert np.isfinite(m0) and m0 < 0
    norm = np.linalg.norm(gf)
    cos = float(ga @ gf / (np.linalg.norm(ga) * norm))
    assert cos >= 0.99, cos
    assert np.max(np.abs(ga - gf)) <= 0.05 * norm, (ga, gf)


def test_autograd_gradcheck(lib):
    torch = pytest.importorskip("torch")
    hol = _case(16)
    cfg = _perturbed(hol, 1)
    h, _ = _handle(lib, cfg, hol.frames)
    assert lib.digHoloB200FreezeWindow(h, 1) == 0
    steps = _steps(lib, h, cfg)
    # all twelve parameters: the locked waist is one parameter (polarisation 0
    # carries the gradient of both)
    params = [(pol, k) for pol in (0, 1) for k in KINDS[:5]] + [(0, "waist")]
    base = [_get(lib, h, pol, k) for pol, k in params]

    class IL(torch.autograd.Function):
        @staticmethod
        def forward(ctx, z):
            for (pol, k), b, zi in zip(params, base, z.tolist()):
                _set(lib, h, pol, k, b + zi * steps[k])
            g, il = _grad(lib, h)
            ctx.save_for_backward(torch.tensor([g[pol, KINDS.index(k)] * steps[k] for pol, k in params],
                                               dtype=torch.float64))
            return torch.tensor(il, dtype=torch.float64)

        @staticmethod
        def backward(ctx, go):
            (gz,) = ctx.saved_tensors
            return go * gz

    z = torch.zeros(len(params), dtype=torch.float64, requires_grad=True)
    ok = torch.autograd.gradcheck(IL.apply, (z,), eps=0.05, atol=5e-3, rtol=5e-2, nondet_tol=1e-4,
                                  raise_exception=False)
    lib.digHoloDestroy(h)
    assert ok


def _align(L, cfg, frames, adjoint, waist=True, goal=0):
    # the second search on the same handle is timed (the first one allocates
    # the handle's buffers); both start from the same perturbed settings
    h, fr = _handle(L, cfg, frames)
    for run in range(2):
        if run:
            api.configure(L, h, cfg)
            b, m, p = C.c_int(), C.c_int(), C.c_int()
            L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
        L.digHoloConfigSetAutoAlignBasisWaist(h, 1 if waist else 0)
        L.digHoloConfigSetAutoAlignMode(h, 1)
        L.digHoloConfigSetAutoAlignGoalIdx(h, goal)
        L.digHoloConfigSetAutoAlignTol(h, 0.01)
        L.digHoloConfigSetAutoAlignFourierWindowRadius(h, 0)
        L.digHoloB200Synchronize(h)
        t = time.perf_counter()
        val = L.digHoloB200AutoAlignAdjoint(h) if adjoint else L.digHoloAutoAlign(h)
        L.digHoloB200Synchronize(h)
        dt = time.perf_counter() - t
    metrics = np.array([L.digHoloAutoAlignGetMetric(h, i) for i in range(9)])
    ev = L.digHoloB200GetAutoAlignEvaluations(h)
    L.digHoloDestroy(h)
    return metrics, dt, ev


@pytest.mark.parametrize("mode", [0, 1])
def test_adjoint_autoalign_matches_plain(lib, mode):
    hol = _case(32)
    cfg = _perturbed(hol, mode)
    waist = mode == 0
    mp, tp, ep = _align(lib, cfg, hol.frames, False, waist)
    ma, ta, ea = _align(lib, cfg, hol.frames, True, waist)
    print("mode %d plain search IL %.4f MDL %.4f in %.1f ms (%d evaluations); adjoint IL %.4f MDL %.4f in %.1f ms (%d)"
          % (mode, mp[0], mp[1], 1e3 * tp, ep, ma[0], ma[1], 1e3 * ta, ea))
    assert ma[0] >= mp[0] - 0.01


def test_adjoint_autoalign_goal_mdl(lib):
    """Goal MDL: the adjoint search (an IL pass, then an MDL pass, as the
    reference's search with goal MDL) reaches at least the plain search's
    MDL, within 0.01 dB, full resolution, on 256 frames (more frames than
    the 240 modes, as in the benchmark's 512; with fewer frames than modes
    the adjoint's MDL has been measured 0.010-0.018 dB short)."""
    hol = _case(256)
    cfg = _perturbed(hol, 0)
    mp, tp, ep = _align(lib, cfg, hol.frames, False, True, goal=1)
    ma, ta, ea = _align(lib, cfg, hol.frames, True, True, goal=1)
    print("goal MDL: plain search IL %.4f MDL %.4f in %.1f ms (%d evaluations); adjoint IL %.4f MDL %.4f in %.1f ms (%d)"
          % (mp[0], mp[1], 1e3 * tp, ep, ma[0], ma[1], 1e3 * ta, ea))
    assert ma[1] >= mp[1] - 0.01
