"""FP64 numpy restatement of digHolo's batch-processing path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it may be imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
digholo_b200 product.

Parity status: pinned against the reference itself.  oracle/Makefile builds
the unmodified reference (digHolo.cpp) into oracle/_ref, and
tests/test_oracle_pin.py runs both on the same synthetic holograms (and on the
committed fixtures in tests/golden/, generated by tests/golden/make_golden.py
from that build).  The reference ships no golden vectors or known-answer
tests of its own.

It restates, step by step, the work of digHoloProcessBatch
(digHolo.cpp:4693-4728):

  fft_windows         FFT window snap/clamp           digHolo.cpp:7267-7378
  k_axes / xy_axes    Fourier and camera axes         digHolo.cpp:2843-2874, 7720-7733
  ifft_windows        IFFT window bounds              digHolo.cpp:7868-8048
  ifft_axes           reconstructed-plane axes        digHolo.cpp:8183-8203
  copy_window         Fourier window copy             digHolo.cpp:1808-2122
  average_windows     frame averaging of windows      digHolo.cpp:8643-8700, 1886-2118
  field_analysis      power / CoM / max / Aeff        digHolo.cpp:2354-2654, 9103-9176
  fourier_analysis    the same on the R2C plane       digHolo.cpp:6931-6980, 8990-9180
  reference_wave      separable tilt/defocus wave     digHolo.cpp:10201-10504
  apply_tilt          -conj(A.ref) and int16 rounding digHolo.cpp:2701-2837
  hg_basis            int16 HG modes and scales       digHolo.cpp:1269-1484, 10543-10645
  overlap             separable HG overlap            digHolo.cpp:2149-2341, 9756-9815
  auto_align_snap     AutoAlign parameter estimate    digHolo.cpp:11517-11970
  auto_focus          its focus search                digHolo.cpp:11181-11499
  dct2_redft          FFTW REDFT10 / REDFT01 (2D)     digHolo.cpp:7393-7420
  ref_cal_store       reference-wave calibration      digHolo.cpp:5419-5555
  ref_cal_planes      its reconstructed planes        digHolo.cpp:6729-6830, 8253-8285

Two flavours are produced by :func:`process_batch`:

* ``quantised``: the reference's own storage formats (int16 fields with scale
  32767/max|E|, 14-bit reference wave, int16 HG modes with per-mode scales),
  emulating its float32 arithmetic where that decides a rounding;
* ``exact``: the same mathematics with no quantisation, everything in FP64
  (the "FP64 oracle" that FP32 GPU results are scored against).

Deliberate difference: the reference applies the overlap's int16->float
scale only inside its ``pixelIdy == pixelCountY - 16`` branch
(digHolo.cpp:2318-2331), so when the reconstructed field is exactly 16 rows
high the scale is never applied and raw integer sums come out.  The
quantised flavour here applies the scale always; ``reference_unscaled_16``
reproduces the reference's behaviour for the pinning test.
"""
import math

import numpy as np

F32 = np.float32
PI_F = F32(3.14159265358979323846264338327950288)  # const float pi, digHolo.cpp:89
PI_D = 3.14159265358979323846264338327950288      # piD, digHolo.cpp:3633
UNIT_ANGLE = F32(PI_F / F32(180.0))                # DIGHOLO_UNIT_ANGLE (pi/180.0f), digHolo.h:192
PIXEL_QUANTA = 16


class Config:
    """The fields of digHoloConfig (digHolo.cpp:3323-3372) that the batch path reads."""

    def __init__(self, frame_width=320, frame_height=256, pixel_size=20e-6, pol_count=1,
                 fft_window=(0, 0), window_radius_deg=0.4, resolution_mode=0,
                 wavelength=1565e-9, beam_centre=None, tilt_deg=None, defocus=None,
                 waist=None, max_mg=0, fill_factor=1, pol_lock_tilt=0, pol_lock_defocus=0,
                 pol_lock_waist=1, avg_count=1, avg_mode=0, batch_cal=None, ref_cal=None):
        self.frame_width = frame_width
        self.frame_height = frame_height
        self.pixel_size = F32(pixel_size)
        self.pol_count = pol_count
        self.fft_window = fft_window
        self.window_radius_deg = F32(window_radius_deg)
        self.resolution_mode = resolution_mode
        self.wavelength = F32(wavelength)
        self.beam_centre = [[F32(0), F32(0)], [F32(0), F32(0)]] if beam_centre is None else \
            [[F32(v) for v in bc] for bc in beam_centre]
        self.tilt_deg = [[F32(-0.75), F32(0.75)], [F32(-0.75), F32(0.75)]] if tilt_deg is None else \
            [[F32(v) for v in t] for t in tilt_deg]
        self.defocus = [F32(0), F32(0)] if defocus is None else [F32(v) for v in defocus]
        self.waist = [F32(510), F32(510)] if waist is None else [F32(v) for v in waist]
        self.max_mg = max_mg
        self.fill_factor = fill_factor
        self.pol_lock_tilt = pol_lock_tilt
        self.pol_lock_defocus = pol_lock_defocus
        self.pol_lock_waist = pol_lock_waist
        self.avg_count = avg_count
        self.avg_mode = avg_mode
        # digHoloConfigSetBatchCalibration: complex (polCount, batchCount) factors
        self.batch_cal = None if batch_cal is None else np.asarray(batch_cal, dtype=np.complex64)
        # digHoloConfigSetRefCalibration*: the stored factors (count, frameHeight,
        # frameWidth) complex, as ref_cal_store forms them
        self.ref_cal = ref_cal
        while len(self.beam_centre) < 2:
            self.beam_centre.append([F32(0), F32(0)])
        while len(self.tilt_deg) < 2:
            self.tilt_deg.append([F32(-0.75), F32(0.75)])
        while len(self.defocus) < 2:
            self.defocus.append(F32(0))
        while len(self.waist) < 2:
            self.waist.append(F32(510))


def _round_half_away(x):
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def fft_windows(cfg):
    """FFT window size and per-polarisation corners (digHolo.cpp:7283-7378)."""
    fx = cfg.fft_window[0] if cfg.fft_window[0] > 0 else cfg.frame_width // cfg.pol_count
    fy = cfg.fft_window[1] if cfg.fft_window[1] > 0 else cfg.frame_height
    W = PIXEL_QUANTA * (fx // PIXEL_QUANTA)
    H = PIXEL_QUANTA * (fy // PIXEL_QUANTA)
    W = max(W, 16)
    H = max(H, 16)
    W = min(W, cfg.frame_width)
    H = min(H, cfg.frame_height)
    block = 16  # ALIGN / sizeof(float), digHolo.cpp:7311
    cxs, cys = [], []
    for pol in range(cfg.pol_count):
        bcx = F32(cfg.beam_centre[pol][0])
        bcy = F32(cfg.beam_centre[pol][1])
        CX = F32(F32(bcx / cfg.pixel_size) + F32(cfg.frame_width // 2))
        CY = F32(F32(bcy / cfg.pixel_size) + F32(cfg.frame_height // 2))
        cx = int(_round_half_away(float(F32(F32(CX - F32(W // 2)) / F32(block))))) * block
        cy = int(_round_half_away(float(F32(CY - F32(H // 2)))))
        cx = max(cx, 0)
        cy = max(cy, 0)
        if cx + W > cfg.frame_width:
            cx = cfg.frame_width - W
        if cy + H > cfg.frame_height:
            cy = cfg.frame_height - H
        cxs.append(cx)
        cys.append(cy)
    return W, H, cxs, cys


def _gen_axis_shifted(n, step):
    return np.array([F32(step) * F32(i if i <= n // 2 else i - n) for i in range(n)], dtype=F32)


def _gen_axis_centred(n, step):
    return np.array([F32(i - n // 2) * F32(step) for i in range(n)], dtype=F32)


def k_axes(W, H, pixel_size):
    """fftshifted kx, ky axes of the FFT plane (digHolo.cpp:7724-7733)."""
    period = F32(2.0 * float(pixel_size))
    kfx = F32(2 * (2.0 * PI_D / float(period)) / W)
    kfy = F32(2 * (2.0 * PI_D / float(period)) / H)
    return _gen_axis_shifted(W, kfx), _gen_axis_shifted(H, kfy)


def xy_axes(W, H, pixel_size):
    """Camera-plane axes of the FFT window (digHolo.cpp:7732)."""
    return _gen_axis_centred(W, pixel_size), _gen_axis_centred(H, pixel_size)


def _tilts_rad(cfg):
    out = []
    for pol in range(cfg.pol_count):
        src = 0 if cfg.pol_lock_tilt else pol
        out.append((F32(cfg.tilt_deg[src][0] * UNIT_ANGLE), F32(cfg.tilt_deg[src][1] * UNIT_ANGLE)))
    return out


def ifft_windows(cfg, W, H, kx, ky, zero_tilt=False):
    """IFFT window size and corners (digHolo.cpp:7868-8048), single wavelength.

    zero_tilt: the calibration's window (no zernCoefs: tilt 0, and a c2c
    plane, so no clamp to the positive kx half; digHolo.cpp:6812-6818)."""
    lam = cfg.wavelength
    k0max = F32(F32(2) * PI_F / lam)
    k0min = k0max
    dkx = F32(kx[1] - kx[0])
    dky = F32(ky[1] - ky[0])
    r0 = F32(cfg.window_radius_deg * UNIT_ANGLE)
    tilts = [(F32(0), F32(0))] * cfg.pol_count if zero_tilt else _tilts_rad(cfg)
    woi_cx, woi_cy, ww, wh = [], [], [], []
    for pol in range(cfg.pol_count):
        tx, ty = tilts[pol]
        maxEX = F32(float(F32(F32(F32(tx + r0) * k0max) / dkx)) + W / 2.0)
        maxEY = F32(float(F32(F32(F32(ty + r0) * k0max) / dky)) + H / 2.0)
        minSX = F32(float(F32(F32(F32(tx - r0) * k0min) / dkx)) + W / 2.0)
        minSY = F32(float(F32(F32(F32(ty - r0) * k0min) / dky)) + H / 2.0)
        woi_cx.append(int(_round_half_away(float(F32(maxEX + minSX)) / 4.0)) * 2)
        woi_cy.append(int(_round_half_away(float(F32(maxEY + minSY)) / 4.0)) * 2)
        wpol = int(F32(F32(maxEX - minSX) + F32(1)))
        hpol = int(F32(F32(maxEY - minSY) + F32(1)))
        wpol = int(F32(16) * F32(math.ceil(float(F32(F32(wpol) / F32(16))))))
        hpol = int(F32(16) * F32(math.ceil(float(F32(F32(hpol) / F32(16))))))
        ww.append(wpol)
        wh.append(hpol)
    w = max(max(ww), 16)
    h = max(max(wh), 16)
    sx, sy = [], []
    for pol in range(cfg.pol_count):
        nsx = int(woi_cx[pol] - w / 2.0)
        if nsx < W // 2 and not zero_tilt:
            nsx = W // 2
        if nsx < 0:
            nsx = 0
        if nsx + w > W:
            nsx = W - w
        nsy = int(woi_cy[pol] - h / 2.0)
        sx.append(nsx)
        sy.append(nsy)
    return w, h, sx, sy


def ifft_axes(cfg, W, H, w, h):
    """Axes of the reconstructed plane (digHolo.cpp:8183-8203)."""
    if cfg.resolution_mode == 0:
        w, h = W, H
    psx = F32(F32(cfg.pixel_size * F32(W)) / F32(w))
    psy = F32(F32(cfg.pixel_size * F32(H)) / F32(h))
    return _gen_axis_centred(w, psx), _gen_axis_centred(h, psy)


def xcsc(x):
    """x / sin(x), 1 at x = 0 (the inverse pixel sinc, digHolo.cpp:820-866)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    nz = x != 0
    out[nz] = x[nz] / np.sin(x[nz])
    return out


def copy_window(F, cfg, pol, W, H, w, h, SX, SY, cx, cy, kx, ky):
    """Fourier-window selection for one polarisation (digHolo.cpp:1808-2122).

    F: (..., H, W/2+1) complex R2C planes.  Returns (..., h, w) in low-res
    mode or (..., H, W) in full-res mode.  Single frame per output
    (avgCount = 1) and no batch calibration.
    """
    lowres = cfg.resolution_mode == 1
    fw, fh = cfg.frame_width, cfg.frame_height
    p = cfg.pixel_size
    cx0 = (cx + W // 2) - fw // 2
    cy0 = (cy + H // 2) - fh // 2
    bcx = float(F32(cfg.beam_centre[pol][0] - F32(F32(cx0) * p)))
    bcy = float(F32(cfg.beam_centre[pol][1] - F32(F32(cy0) * p)))
    src = 0 if cfg.pol_lock_tilt else pol
    # digHolo.cpp:8588-8589, 8627-8630 (per-polarisation tilt, sin of the angle)
    tx = F32(cfg.tilt_deg[pol][0] * UNIT_ANGLE)
    ty = F32(cfg.tilt_deg[pol][1] * UNIT_ANGLE)
    del src
    k0_f = F32(F32(2) * PI_F / cfg.wavelength)
    kx0_f = F32(k0_f * F32(math.sin(float(tx))))
    ky0_f = F32(k0_f * F32(math.sin(float(ty))))
    kr_f = F32(k0_f * F32(math.sin(float(F32(cfg.window_radius_deg * UNIT_ANGLE)))))
    r02_f = F32(kr_f * kr_f)
    ifft_len = (w * h) if lowres else (W * H)
    norm = 1.0 / math.sqrt(float(W * H) * float(ifft_len))
    shape = F.shape[:-2]
    out = np.zeros(shape + ((h, w) if lowres else (H, W)), dtype=np.complex128)
    ky_shift = abs(float(ky[1] - ky[0]) * H)
    SX0 = SX - W // 2
    cols = np.arange(w) + SX0
    kxv = kx[cols].astype(np.float64)
    sinc_x = xcsc(kxv * (0.5 * float(p))) if cfg.fill_factor else np.ones(w)
    for j in range(h):
        jsy = j + SY
        row = (jsy + H // 2) % H
        kyv = float(ky[row])
        shift = ky_shift if jsy < 0 else (-ky_shift if jsy > H else 0.0)
        # the mask test in float32, as digHolo.cpp:2006-2019 evaluates it
        dky = F32(F32(ky[row]) - F32(ky0_f + F32(shift)))
        dkx = (kx[cols] - kx0_f).astype(F32)
        dr2 = (dkx * dkx).astype(F32) + F32(dky * dky)
        inside = dr2.astype(F32) <= r02_f
        env = sinc_x * (xcsc(np.array([kyv * 0.5 * float(p)]))[0] if cfg.fill_factor else 1.0)
        adj = np.where(inside, norm * env, 0.0) * np.exp(1j * (kxv * bcx + kyv * bcy))
        vals = F[..., row, cols] * adj
        if lowres:
            out[..., j, :] = vals
        else:
            out[..., row, cols % W] = vals
    return out


def field_analysis(E, x, y):
    """Per-field statistics over the whole plane (digHolo.cpp:2354-2654 with
    windowRadius = 0, aggregated as in digHolo.cpp:9103-9176).

    E: (B, h, w) complex.  Returns a dict of (B+1,) arrays; entry B is the
    analysis of the intensity summed over the batch.  MAXABS is stored as
    32767 / max|E| like the reference.
    """
    B, ny, nx = E.shape
    I = (np.abs(E) ** 2) / (nx * ny)
    Isum = np.cumsum(I, axis=0)[-1:]
    allI = np.concatenate([I, Isum], axis=0)
    X = x.astype(np.float64)[None, None, :]
    Y = y.astype(np.float64)[None, :, None]
    P = allI.sum(axis=(1, 2))
    comx = (allI * X).sum(axis=(1, 2)) / P
    comy = (allI * Y).sum(axis=(1, 2)) / P
    E4 = (allI ** 2).sum(axis=(1, 2))
    dA = abs(float(x[2] - x[1])) * abs(float(y[2] - y[1]))
    aeff = dA * P * P / E4
    mx = np.sqrt(np.concatenate([(np.abs(E) ** 2).reshape(B, -1).max(axis=1),
                                 [allI.reshape(B + 1, -1)[-1].max()]]))
    return {"power": P, "comx": comx, "comy": comy, "aeff": aeff, "maxabs": mx,
            "scale": np.array([float(F32(32767.0 / m)) if m > 0 else np.inf for m in mx])}


def fourier_analysis(F, kx, ky, wavelength, aperture_deg):
    """FFT-stage analysis of one polarisation's R2C planes (digHoloFFTAnalysis,
    digHolo.cpp:6931-6980 -> digHoloFieldAnalysisRoutine 8990-9180 ->
    digHoloFieldAnalysis 2354-2654 with removeZeroOrder1D set and no y wrap).

    F: (B, H, W/2+1) complex R2C planes.  As the reference does, the plane's
    column i and row j are given the fftshifted axis values kx[i], ky[j].
    Pixel (j, i) enters when j is neither 0 nor H/2, 0 < i < 8 floor(Nx/8)
    (Nx = W/2+1), and kx[i]^2 + ky[j]^2 >= R^2 with R = 2 k0 sin(aperture)
    (float32); the other pixels count as zero.  Intensity I = |F|^2/(Nx Ny).
    Returns per-frame and batch-sum statistics ((B+1,) arrays: power, comx,
    comy, comywrap, aeff, maxabs, scale = 32767/maxabs, maxidx = 2 j Nx + i of
    the maximum, the larger index on ties, plus 8 for the batch-sum entry as
    the reference reads it) and the batch-sum plane (H, Nx).
    The per-frame maximum is of |F| (unnormalised), the batch entry's of the
    summed normalised intensity, as in the reference.
    """
    F = np.asarray(F)
    B, Ny, Nx = F.shape
    k0 = F32(F32(2) * PI_F / F32(wavelength))
    R = F32(F32(2) * k0 * F32(np.sin(F32(F32(aperture_deg) * UNIT_ANGLE))))
    xs = kx[:Nx].astype(F32)
    ys = ky[:Ny].astype(F32)
    rx = (xs.astype(F32) * xs.astype(F32)).astype(F32)
    ry = (ys.astype(F32) * ys.astype(F32)).astype(F32)
    rr = (ry[:, None] + rx[None, :]).astype(F32)
    mask = rr >= F32(R * R) if R != 0 else np.ones((Ny, Nx), dtype=bool)
    nxr = 8 * (Nx // 8)
    mask[:, nxr:] = False
    mask[:, 0] = False
    mask[0, :] = False
    mask[Ny // 2, :] = False
    I0 = (np.abs(F) ** 2) * mask[None]
    I = I0 / (Nx * Ny)
    S = I.sum(axis=0)
    allI = np.concatenate([I, S[None]], axis=0)
    X = xs.astype(np.float64)[None, None, :]
    Y = ys.astype(np.float64)[None, :, None]
    shift = abs(float(F32((ys[1] - ys[0]) * F32(Ny))))
    Yw = Y + shift * (Y < 0)
    P = allI.sum(axis=(1, 2))
    with np.errstate(invalid="ignore", divide="ignore"):
        comx = (allI * X).sum(axis=(1, 2)) / P
        comy = (allI * Y).sum(axis=(1, 2)) / P
        comyw = (allI * Yw).sum(axis=(1, 2)) / P
        E4 = (allI ** 2).sum(axis=(1, 2))
        dA = abs(float(kx[2] - kx[1])) * abs(float(ky[2] - ky[1]))
        aeff = dA * P * P / E4
    peak = np.concatenate([I0, S[None]], axis=0).reshape(B + 1, -1)
    flat = np.arange(Ny * Nx)
    idx2 = 2 * (flat // Nx) * Nx + (flat % Nx)
    maxidx = np.array([int(idx2[np.flatnonzero(p == p.max())[-1]]) for p in peak])
    # the batch-sum comparison reads the index vector after it has advanced to
    # the next block of 8 (digHolo.cpp:2533-2561)
    maxidx[-1] += 8
    mx = np.sqrt(peak.max(axis=1))
    with np.errstate(divide="ignore"):
        scale = np.array([float(F32(32767.0 / m)) if m > 0 else np.inf for m in mx])
    return {"power": P, "comx": comx, "comy": comy, "comywrap": comyw, "aeff": aeff, "maxabs": mx,
            "scale": scale, "maxidx": maxidx, "batchsum": S}


def _safe_stats(E, x, y):
    with np.errstate(invalid="ignore", divide="ignore"):
        return field_analysis(E, x, y)


def reference_wave(cfg, pol, x, y, W, H, SX, SY, dkx, dky, quantised=True):
    """Separable reference wave for one polarisation (digHolo.cpp:10201-10504).

    Returns (refX, refY) complex arrays.  With ``quantised`` the values are
    the reference's 14-bit integers (scale 16383) as complex int pairs;
    otherwise exact unit-modulus FP64 values.
    """
    src_t = 0 if cfg.pol_lock_tilt else pol
    src_d = 0 if cfg.pol_lock_defocus else pol
    tx = F32(cfg.tilt_deg[src_t][0] * UNIT_ANGLE)
    ty = F32(cfg.tilt_deg[src_t][1] * UNIT_ANGLE)
    offx = F32(0)
    offy = F32(0)
    if cfg.resolution_mode == 1:
        offx = F32((SX[src_t] - W / 2.0 - 0) * float(dkx))
        offy = F32((SY[src_t] - H / 2.0) * float(dky))
    dioptre = cfg.defocus[src_d]
    lam = cfg.wavelength
    k0 = F32(2.0 * float(PI_F) / float(lam))
    kxv = F32(F32(-k0 * tx) + offx)
    kyv = F32(F32(-k0 * ty) + offy)
    kx0 = kxv if offx == 0 else F32(k0 * F32(-tx))
    ky0 = kyv if offy == 0 else F32(k0 * F32(-ty))
    focal = F32(F32(-PI_F * dioptre) / lam)
    cxp = F32(cfg.beam_centre[pol][0])
    cyp = F32(cfg.beam_centre[pol][1])
    out = []
    for axis, k, piston in ((x, kxv, F32(cxp * kx0)), (y, kyv, F32(cyp * ky0))):
        r = axis.astype(F32)
        if quantised:
            kr = (k.astype(np.float64) * r.astype(np.float64) + float(piston)).astype(F32)  # fmadd
            arg = (kr + (focal * (r * r)).astype(F32)).astype(F32)
            c = np.cos(arg.astype(np.float64)).astype(F32)
            s = np.sin(arg.astype(np.float64)).astype(F32)
            re = np.clip(np.rint((F32(16383.0) * c).astype(F32)), -32768, 32767).astype(np.int32)
            im = np.clip(np.rint((F32(16383.0) * s).astype(F32)), -32768, 32767).astype(np.int32)
            out.append(re + 1j * im)
        else:
            arg = float(k) * r.astype(np.float64) + float(piston) + float(focal) * r.astype(np.float64) ** 2
            out.append(np.exp(1j * arg))
    return out[0], out[1]


def apply_tilt(E, refx, refy, scale, quantised=True):
    """V = -conj(A . refX . refY) and int16 rounding (digHolo.cpp:2701-2837).

    E: (B, h, w) complex; scale: (B,) float32 scales 32767/max|E|.
    Returns (V complex FP64 before rounding, R int16, I int16).
    """
    if quantised:
        xr, xi = refx.real.astype(np.int64), refx.imag.astype(np.int64)
        yr, yi = refy.real.astype(np.int64), refy.imag.astype(np.int64)
        adj_r = (yr[:, None] * xr[None, :] - yi[:, None] * xi[None, :]).astype(F32)
        adj_i = (yr[:, None] * xi[None, :] + yi[:, None] * xr[None, :]).astype(F32)
        k = F32(1.0 / (16383.0 * 16383.0))
        adj = (adj_r * k).astype(np.float64) + 1j * (adj_i * k).astype(np.float64)
    else:
        adj = refy[:, None] * refx[None, :]
    V = -np.conj(E * adj[None])
    sc = np.asarray(scale, dtype=np.float64)[:, None, None]
    with np.errstate(invalid="ignore", over="ignore"):
        r = np.rint(V.real * sc)
        i = np.rint(V.imag * sc)
    # a field with no power has scale 32767/0 = inf; the reference's
    # float->int32 conversion then yields INT_MIN, saturated to -32768
    bad_r = ~np.isfinite(r)
    bad_i = ~np.isfinite(i)
    r[bad_r] = -32768
    i[bad_i] = -32768
    R = np.clip(r, -32768, 32767).astype(np.int16)
    I = np.clip(i, -32768, 32767).astype(np.int16)
    return V, R, I


def hg_modes(axis, w0, count):
    """Unit-power HG modes on a float32 axis as digHolo builds them
    (digHolo.cpp:1269-1433): dX from the axis end points, u = sqrt(2) x / w0,
    HG_m = sqrt(dX / w0) * 2^(1/4) * psi_m(u), psi_m the normalised Hermite
    function (FP64 three-term recurrence, digHolo.cpp:1345-1388)."""
    ax = axis.astype(np.float64)
    L = ax.size
    dX = abs((ax[L - 1] - ax[0]) / (L - 1))
    W0 = float(w0)
    # u as the reference forms it: the first four axis samples scaled, then
    # advanced four samples at a time by 4*dX*sqrt(2)/w0 (digHolo.cpp:1287-1294)
    step = 4.0 * dX * (math.sqrt(2) / W0)
    lanes = (math.sqrt(2.0) / W0) * ax[:4]
    blocks = np.concatenate([[0.0], np.cumsum(np.full(L // 4 - 1, step))]) if L >= 8 else np.zeros(L // 4)
    u = (lanes[None, :] + blocks[:, None]).reshape(-1)
    if u.size < L:
        u = math.sqrt(2.0) / W0 * ax
    norm = (1.0 / math.sqrt(W0)) * math.sqrt(dX) / math.sqrt(math.sqrt(0.5))
    modes = np.zeros((count, L))
    g = np.exp(-0.5 * u * u)
    h0 = 0.7511255444649425 * g  # pi^-0.25
    modes[0] = h0
    if count > 1:
        modes[1] = 1.0622519320271970 * u * g  # sqrt(2) pi^-0.25
    for n in range(2, count):
        modes[n] = math.sqrt(2.0 / n) * u * modes[n - 1] - math.sqrt((n - 1.0) / n) * modes[n - 2]
    return modes * norm


def quantise_modes(modes):
    """int16 modes and scales (digHolo.cpp:1436-1471): scale 32767/max|mode|,
    float32 multiply, round half to even, saturating pack."""
    mx = np.abs(modes).max(axis=1)
    sf = 32767.0 / mx
    q = np.clip(np.rint((modes.astype(F32) * sf.astype(F32)[:, None]).astype(F32)), -32768, 32767)
    return q.astype(np.int16), (1.0 / sf).astype(F32)


def basis_axes_modes(cfg, pol, xax, yax, quantised=True):
    """HG modes along x and y for one polarisation (digHolo.cpp:10506-10645).

    Square pixels: one set of modes on the longer axis; the shorter axis uses
    its centred sub-range.  Returns (Hx, Hy, sx, sy) with Hx (G, nx), Hy (G, ny).
    """
    G = cfg.max_mg
    w0 = cfg.waist[0] if (cfg.pol_lock_waist or pol == 0) else cfg.waist[pol]
    if w0 == 0:
        w0 = F32(400e-6)
    psx = F32(xax[1] - xax[0])
    psy = F32(yax[1] - yax[0])
    nx, ny = xax.size, yax.size
    if psx == psy:
        long_ax = xax if nx >= ny else yax
        m = hg_modes(long_ax, w0, G)
        if quantised:
            q, s = quantise_modes(m)
        else:
            q, s = m, np.ones(G, dtype=F32)
        L = long_ax.size
        off = (L - min(nx, ny)) // 2
        if nx >= ny:
            return q[:, :nx], q[:, off:off + ny], s, s
        return q[:, off:off + nx], q[:, :ny], s, s
    mx = hg_modes(xax, w0, G)
    my = hg_modes(yax, w0, G)
    if quantised:
        qx, sx = quantise_modes(mx)
        qy, sy = quantise_modes(my)
        return qx, qy, sx, sy
    return mx, my, np.ones(G, dtype=F32), np.ones(G, dtype=F32)


def hg_index(max_mg):
    """Mode enumeration (digHolo.cpp:1245-1265): list of (m, n) per mode index."""
    out = []
    for g in range(max(max_mg, 1)):
        for k in range(g + 1):
            out.append((g - k, k))
    return out


def overlap(R, I, Hx, Hy, sx, sy, field_scale, max_mg, quantised=True):
    """Separable overlap c_mn = sum_y Hy_n(y) sum_x Hx_m(x) F(x, y)
    (digHolo.cpp:2149-2341), no conjugation.  R, I: (B, h, w) int16 (or
    float) field; field_scale: (B,) multiplier to real units.  Returns (B, M)."""
    idx = hg_index(max_mg)
    if quantised:
        Fr = R.astype(np.int64)
        Fi = I.astype(np.int64)
        Tx_r = np.einsum("byx,mx->bym", Fr, Hx.astype(np.int64))
        Tx_i = np.einsum("byx,mx->bym", Fi, Hx.astype(np.int64))
        Cr = np.einsum("bym,ny->bmn", Tx_r, Hy.astype(np.int64)).astype(np.float64)
        Ci = np.einsum("bym,ny->bmn", Tx_i, Hy.astype(np.int64)).astype(np.float64)
    else:
        Cr = np.einsum("byx,mx,ny->bmn", R, Hx, Hy)
        Ci = np.einsum("byx,mx,ny->bmn", I, Hx, Hy)
    out = np.zeros((R.shape[0], len(idx)), dtype=np.complex128)
    fs = np.asarray(field_scale, dtype=np.float64)
    for k, (m, n) in enumerate(idx):
        s = float(sx[m]) * float(sy[n])
        out[:, k] = (Cr[:, m, n] + 1j * Ci[:, m, n]) * s * fs
    return out


def batch_factors(cfg, pol, batch):
    """Batch calibration factor of each batch item of one polarisation:
    cal[pol % calPolCount][item % calBatchCount] (digHolo.cpp:8443-8448,
    8636-8641), or None when no calibration is set."""
    cal = getattr(cfg, "batch_cal", None)
    if cal is None:
        return None
    row = cal[pol % cal.shape[0]]
    return np.array([complex(row[b % cal.shape[1]]) for b in range(batch)])


def average_windows(win, batch, avg, mode, lowres, W, H, w, h, SX, SY, cal=None):
    """Frame averaging of the Fourier windows (digHolo.cpp:8643-8700 and the
    two-pass branch of digHoloCopyWindow, digHolo.cpp:1886-1932, 2062-2118).

    win: (batch * avg, ...) windows of one polarisation in frame order.
    Frames of batch item b: b * avg + k (mode 0, sequential), k * batch + b
    (mode 1, interlaced), b + k (mode 2 with one wavelength, as the
    reference's formula gives).  The first is scaled by 1/avg; each further
    window is multiplied by the unit phase of sum(acc * conj(window)) over the
    window pixels and by 1/avg, and added.  In full-resolution mode only the
    window's pixels enter the correlation, as in the reference.  ``cal``
    (one factor per batch item) multiplies every window of its item as it is
    copied (digHolo.cpp:1831-1835, 2007-2008).
    """
    out = np.zeros((batch,) + win.shape[1:], dtype=np.complex128)
    if lowres:
        sel = (slice(None), slice(None))
    else:
        rows = (np.arange(h) + SY + H // 2) % H
        cols = (np.arange(w) + SX - W // 2) % W
        sel = (rows[:, None], cols[None, :])
    for b in range(batch):
        for k in range(avg):
            f = b * avg + k if mode == 0 else (k * batch + b if mode == 1 else b + k)
            wf = win[f] if cal is None else win[f] * cal[b]
            if k == 0:
                out[b] = wf / avg
            else:
                c = np.sum(out[b][sel] * np.conj(wf[sel]))
                out[b] = out[b] + wf * (c / abs(c)) / avg
    return out


def ref_cal_store(intensity=None, field=None):
    """The factors the reference stores for a reference-wave calibration
    (digHolo.cpp:5419-5555), in float32: from uint16 intensities I,
    sqrt(1 / (I / max I)); from complex fields E, the componentwise
    (1 / (re / max|E|), -1 / (im / max|E|)) -- not the complex inverse --
    with both parts 0 where either is NaN or infinite.  Returns complex64
    (count, height, width)."""
    if intensity is not None:
        I = np.asarray(intensity, dtype=np.uint16)
        scale = F32(F32(1.0) / F32(int(I.max())))
        with np.errstate(divide="ignore", invalid="ignore"):
            v = (F32(1.0) / (I.astype(F32) * scale)).astype(F32)
        v[~np.isfinite(v)] = 0
        return np.sqrt(v).astype(F32).astype(np.complex64)
    E = np.asarray(field, dtype=np.complex64)
    re, im = E.real.astype(F32), E.imag.astype(F32)
    mx = F32(np.sqrt(F32((re * re + im * im).astype(F32).max())))
    scale = F32(F32(1.0) / mx)
    with np.errstate(divide="ignore", invalid="ignore"):
        vr = (F32(1.0) / (re * scale)).astype(F32)
        vi = (F32(-1.0) / (im * scale)).astype(F32)
    bad = ~(np.isfinite(vr) & np.isfinite(vi))
    vr[bad] = 0
    vi[bad] = 0
    return (vr + 1j * vi).astype(np.complex64)


def ref_cal_planes(cfg):
    """The reconstructed calibration planes (count, P, ny, nx) that multiply
    the IFFT output of every frame before the field analysis and the tilt
    removal (digHolo.cpp:8736-8758), one wavelength.

    Each stored calibration frame goes through the batch path with the
    frames' FFT windows, as a complex frame: a c2c FFT of each
    polarisation's window (digHolo.cpp:6729-6784), the Fourier window at
    zero tilt with no beam-centre phase -- the window placed around kx = ky = 0,
    the aperture mask centred there, the inverse pixel sinc, the batch
    calibration of item `count index`, and the normalisation
    sqrt(res / (W H)) / sqrt(W H ifftLength) (digHolo.cpp:8253-8285, and
    digHoloCopyWindow's c2c branches, digHolo.cpp:1808-2122) -- and an
    unnormalised IFFT of the field's size.  Low resolution places the window
    fftshifted into an h x w plane, full resolution at its own frequencies in
    the H x W plane."""
    cal = np.asarray(cfg.ref_cal)
    count = cal.shape[0]
    P = cfg.pol_count
    lowres = cfg.resolution_mode == 1
    W, H, cxs, cys = fft_windows(cfg)
    kx, ky = k_axes(W, H, cfg.pixel_size)
    w, h, _, _ = ifft_windows(cfg, W, H, kx, ky)
    _, _, SXc, SYc = ifft_windows(cfg, W, H, kx, ky, zero_tilt=True)
    nx, ny = (w, h) if lowres else (W, H)
    norm0 = F32(np.sqrt(F32((1.0 * nx * ny) / (1.0 * W * H))))
    ifft_len = (w * h) if lowres else (W * H)
    norm = float(F32(float(norm0) / math.sqrt(float(W * H) * float(ifft_len))))
    k0 = F32(F32(2) * PI_F / cfg.wavelength)
    kr = F32(k0 * F32(math.sin(float(F32(cfg.window_radius_deg * UNIT_ANGLE)))))
    r02 = F32(kr * kr)
    ky_shift = abs(float(ky[1] - ky[0]) * H)
    hp = 0.5 * float(cfg.pixel_size)
    out = np.zeros((count, P, ny, nx), dtype=np.complex128)
    i = np.arange(w)
    for c in range(count):
        for pol in range(P):
            F = np.fft.fft2(cal[c, cys[pol]:cys[pol] + H, cxs[pol]:cxs[pol] + W].astype(np.complex128))
            bf = 1.0
            if getattr(cfg, "batch_cal", None) is not None:
                bc = cfg.batch_cal
                bf = complex(bc[pol % bc.shape[0]][c % bc.shape[1]])
            plane = np.zeros((ny, nx), dtype=np.complex128)
            col = i + SXc[pol] - W // 2
            col = np.where(col < 0, col + W, col)
            ok = (col >= 0) & (col < W)
            colc = np.clip(col, 0, W - 1)
            kxv = kx[colc]
            env_x = xcsc(kxv.astype(np.float64) * hp) if cfg.fill_factor else np.ones(w)
            for j in range(h):
                jsy = j + SYc[pol]
                row = (jsy + H // 2) % H
                shift = ky_shift if jsy < 0 else (-ky_shift if jsy > H else 0.0)
                dky = F32(F32(ky[row]) - F32(F32(0) + F32(shift)))
                dr2 = (kxv * kxv).astype(F32) + F32(dky * dky)
                inside = (dr2.astype(F32) <= r02) & ok
                env = env_x * (xcsc(np.array([float(ky[row]) * hp]))[0] if cfg.fill_factor else 1.0)
                vals = np.where(inside, F[row, colc] * bf * norm * env, 0.0)
                if lowres:
                    plane[(j + h // 2) % h, (i + w // 2) % w] = vals
                else:
                    plane[row, colc[ok]] = vals[ok]
            out[c, pol] = np.fft.ifft2(plane) * (nx * ny)
    return out


def r2c_windows(frames, cfg, W, H, cxs, cys):
    """FP64 R2C of each polarisation's FFT window: (B, P, H, W/2+1)."""
    f = np.asarray(frames, dtype=np.float64)
    out = []
    for pol in range(cfg.pol_count):
        win = f[:, cys[pol]:cys[pol] + H, cxs[pol]:cxs[pol] + W]
        out.append(np.fft.rfft2(win))
    return np.stack(out, axis=1)


def process_batch(frames, cfg, quantised=True):
    """Run the batch path on ``frames`` (B, frameHeight, frameWidth).

    Returns a dict with: geometry, ``window`` (B, P, h, w) Fourier windows,
    ``field_untilted`` (B, P, ny, nx), ``field`` (B, P, ny, nx) complex
    (quantised: int16 x 1/scale, like digHoloGetFields), ``R``/``I`` int16,
    ``scale`` (B, P), ``coefs`` (B, P, M), ``stats`` per polarisation.
    """
    frames = np.asarray(frames)
    avg = int(getattr(cfg, "avg_count", 1) or 1)
    B = frames.shape[0] // avg
    P = cfg.pol_count
    W, H, cxs, cys = fft_windows(cfg)
    kx, ky = k_axes(W, H, cfg.pixel_size)
    w, h, SX, SY = ifft_windows(cfg, W, H, kx, ky)
    xax, yax = ifft_axes(cfg, W, H, w, h)
    nx, ny = xax.size, yax.size
    Fplanes = r2c_windows(frames, cfg, W, H, cxs, cys)
    cal_planes = None
    rc = getattr(cfg, "ref_cal", None)
    if rc is not None and rc.shape[1] == cfg.frame_height and rc.shape[2] == cfg.frame_width:
        cal_planes = ref_cal_planes(cfg)
    res = {"W": W, "H": H, "cx": cxs, "cy": cys, "w": w, "h": h, "SX": SX, "SY": SY,
           "x": xax, "y": yax, "kx": kx, "ky": ky, "fourier": Fplanes,
           "fft_stats": [fourier_analysis(Fplanes[:, p], kx, ky, cfg.wavelength, cfg.window_radius_deg)
                         for p in range(P)]}
    windows = np.zeros((B, P, h if cfg.resolution_mode else H, w if cfg.resolution_mode else W),
                       dtype=np.complex128)
    untilted = np.zeros((B, P, ny, nx), dtype=np.complex128)
    field = np.zeros((B, P, ny, nx), dtype=np.complex128)
    field_v = np.zeros((B, P, ny, nx), dtype=np.complex128)
    Rs = np.zeros((B, P, ny, nx), dtype=np.int16)
    Is = np.zeros((B, P, ny, nx), dtype=np.int16)
    scales = np.zeros((B, P))
    stats = []
    M = len(hg_index(cfg.max_mg)) if cfg.max_mg > 0 else 0
    coefs = np.zeros((B, P, M), dtype=np.complex128)
    for pol in range(P):
        win = copy_window(Fplanes[:, pol], cfg, pol, W, H, w, h, SX[pol], SY[pol], cxs[pol], cys[pol], kx, ky)
        cal = batch_factors(cfg, pol, B)
        if avg > 1:
            win = average_windows(win, B, avg, int(getattr(cfg, "avg_mode", 0)), cfg.resolution_mode == 1,
                                  W, H, w, h, SX[pol], SY[pol], cal)
        elif cal is not None:
            win = win * cal[:, None, None]
        windows[:, pol] = win
        E = np.fft.ifft2(win) * (win.shape[-1] * win.shape[-2])
        if cal_planes is not None:
            E = E * cal_planes[0, pol]
        untilted[:, pol] = E
        st = _safe_stats(E, xax, yax)
        stats.append(st)
        scale = st["scale"][:B]
        scales[:, pol] = scale
        refx, refy = reference_wave(cfg, pol, xax, yax, W, H, SX, SY, kx[1] - kx[0], ky[1] - ky[0], quantised)
        V, R, I = apply_tilt(E, refx, refy, scale, quantised)
        field_v[:, pol] = V
        Rs[:, pol] = R
        Is[:, pol] = I
        if quantised:
            inv = np.array([float(F32(1.0 / s)) if np.isfinite(s) else 0.0 for s in scale])
            field[:, pol] = (R.astype(np.float64) + 1j * I.astype(np.float64)) * inv[:, None, None]
        else:
            field[:, pol] = V
        if M:
            Hx, Hy, sx, sy = basis_axes_modes(cfg, pol, xax, yax, quantised)
            if quantised:
                fs = np.array([float(F32(F32(1.0) / F32(s))) if np.isfinite(s) else 0.0 for s in scale])
                coefs[:, pol] = overlap(R, I, Hx, Hy, sx, sy, fs, cfg.max_mg, True)
            else:
                coefs[:, pol] = overlap(V.real, V.imag, Hx, Hy, sx, sy, np.ones(B), cfg.max_mg, False)
    res.update(window=windows, field_untilted=untilted, field=field, field_v=field_v,
               R=Rs, I=Is, scale=scales, coefs=coefs, stats=stats)
    if M:
        res["coefs_out"] = transform_coefs(coefs, cfg)
    return res


# ---------------------------------------------------------------- basis transforms

def lg_transform(G):
    """HG -> LG transform of the modes of G groups, (M, M) complex with
    T[i, j] the weight of HG mode i in LG mode j (digHoloLGInit,
    digHolo.cpp:9909-10040, and digHoloLGtoHGcoef, digHolo.cpp:9819-9907,
    the Beijersbergen mode-converter expansion).  Group g holds HG (g - c, c)
    at position c and LG l = g - 2r, p = (g - |l|) / 2 at position r.  With
    (n, m) = (p, p - l) for l < 0, else (l + p, p), the weight of HG (hm, hn) is
    [t^hm] (1 + t)^n (1 - t)^m * sqrt(hm! hn! / (n! m! 2^g)) * i^(g + hm),
    negated for odd g and l > 0.  Computed in FP64 and rounded to complex64,
    as the reference stores it."""
    M = G * (G + 1) // 2
    T = np.zeros((M, M), dtype=np.complex128)
    base = 0
    for g in range(G):
        for r in range(g + 1):
            l = g - 2 * r
            p = (g - abs(l)) // 2
            n, m = (p, p - l) if l < 0 else (l + p, p)
            poly = np.array([1.0])
            for _ in range(n):
                poly = np.convolve(poly, [1.0, 1.0])
            for _ in range(m):
                poly = np.convolve(poly, [1.0, -1.0])
            for c in range(g + 1):
                hm, hn = g - c, c
                puv = poly[hm] if hm < poly.size else 0.0
                b = math.sqrt(math.factorial(hm) * math.factorial(hn) / (math.factorial(n) * math.factorial(m)))
                v = puv * b * 2.0 ** (-0.5 * g)
                if g % 2 and l > 0:
                    v = -v
                T[base + c, base + r] = v * (1j ** ((g + hm) % 4))
        base += g + 1
    return T.astype(np.complex64).astype(np.complex128)


def basis_matrix(cfg, M):
    """The active transform (digHoloApplyBasisTransform, digHolo.cpp:9469-9562):
    None for HG (type 0, an unknown type, or an invalid custom matrix), the LG
    matrix for type 1, for type 2 the leading min(M, in) x min(M, out) block of
    the custom [in][out] matrix."""
    t = int(getattr(cfg, "basis_type", 0) or 0)
    if t == 1:
        G = int(round((math.sqrt(8 * M + 1) - 1) / 2))
        return lg_transform(G)
    if t == 2:
        full = getattr(cfg, "basis_custom", None)
        if full is None or full.size == 0:
            return None
        full = np.asarray(full, dtype=np.complex64).astype(np.complex128)
        return full[:min(M, full.shape[0]), :min(M, full.shape[1])]
    return None


def transform_coefs(coefs, cfg):
    """Coefficients in the configured basis: (B, P, modeCountOut), each
    polarisation's HG coefficients times the transform (applyBasisTransform /
    HGtoLG, digHolo.cpp:5000-5037, 9565-9600: no conjugation)."""
    B, P, M = coefs.shape
    T = basis_matrix(cfg, M)
    if T is None:
        return coefs
    return np.einsum("bpi,ij->bpj", coefs[:, :, :T.shape[0]], T)


def reference_unscaled_16(coefs, cfg, res):
    """What digHoloProcessBatch returns when the field is 16 rows high: the
    overlap without its final scale (digHolo.cpp:2318-2331).  Divides the
    properly scaled quantised coefficients by that scale."""
    xax, yax = res["x"], res["y"]
    out = np.array(coefs, copy=True)
    idx = hg_index(cfg.max_mg)
    for pol in range(cfg.pol_count):
        _, _, sx, sy = basis_axes_modes(cfg, pol, xax, yax, True)
        fs = np.array([float(F32(F32(1.0) / F32(s))) for s in res["scale"][:, pol]])
        for k, (m, n) in enumerate(idx):
            out[:, pol, k] = out[:, pol, k] / (float(sx[m]) * float(sy[n]) * fs)
    return out


# ---------------------------------------------------------------- metrics

def power_meter(coefs, pol_independent=False, goal_uses_svd=True):
    """IL / MDL of the batch coefficient matrix (digHolo.cpp:10714-11130) for
    a single wavelength, batchCount > 1, basis output modes.

    coefs: (B, P, M) complex.  Returns dict with linear 'il', 'mdl' from the
    SVD path (used when the goal is MDL and for reported metrics) and
    'il_frob' from the Frobenius path (insertionLoss256, digHolo.cpp:3105-3143),
    plus their values in dB (10 log10, digHolo.cpp:12188).
    """
    B, P, M = coefs.shape
    independent = pol_independent or P == 1
    mats = []
    if P == 1 or not independent:
        mats.append(coefs.reshape(B, P * M).T)       # (modes, batch)
    else:
        for pol in range(P):
            mats.append(coefs[:, pol, :].T)
    svals = []
    for A in mats:
        svals.append(np.linalg.svd(A, compute_uv=False))
    s = np.concatenate(svals)
    il = float(np.mean(s ** 2))
    mdl = float(s.min() ** 2 / s.max() ** 2)
    il_frob = float(sum((np.abs(A) ** 2).sum() / B for A in mats))
    return {"il": il, "mdl": mdl, "il_frob": il_frob,
            "il_db": 10 * math.log10(il), "mdl_db": 10 * math.log10(mdl),
            "il_frob_db": 10 * math.log10(il_frob)}


# ---------------------------------------------------------------- AutoAlign snap (parameter estimate)

def dct2_redft(a, kind):
    """2D FFTW REDFT10 (kind 2, DCT-II) or REDFT01 (kind 3, DCT-III),
    unnormalised, as FFTW defines them: along the last axis, then the first,
    FP64 inside, float32 out (the digHoloDCTPlan / digHoloIDCTPlan pair,
    digHolo.cpp:7393-7420).
      REDFT10: Y_k = 2 sum_j X_j cos(pi (j + 1/2) k / n)
      REDFT01: Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (k + 1/2) / n)
    """
    x = np.asarray(a, dtype=np.float64)

    def mat(n):
        k = np.arange(n)[:, None]
        j = np.arange(n)[None, :]
        if kind == 2:
            return 2.0 * np.cos(np.pi * ((2 * j + 1) * k % (4 * n)) / (2.0 * n))
        m = np.cos(np.pi * ((j * (2 * k + 1)) % (4 * n)) / (2.0 * n)) * 2.0
        m[:, 0] = 1.0
        return m
    y = x @ mat(x.shape[1]).T
    y = mat(x.shape[0]) @ y
    return y.astype(F32)


def snap_filter(out, k0, aperture_rad, pixel_size):
    """The Gaussian filter of the snap's correlation (digHolo.cpp:11611-11643)
    applied as the reference applies it: in blocks of 8 floats per row of
    8 floor(Nx/8) columns, stepping through the (H, Nx) array without its row
    stride, so flat position f gets the factor of row f // (8 floor(Nx/8)) and
    column f % (8 floor(Nx/8)), and the last H floats are left as they are."""
    H, Nx = out.shape
    nb = 8 * (Nx // 8)
    aperturek = F32(k0 * F32(aperture_rad))
    wx = F32((1.0 * math.pi / float(aperturek)) * math.sqrt(2.0))
    wy = F32((2.0 * math.pi / float(aperturek)) * math.sqrt(2.0))
    wx2 = F32(-1.0 / (float(wx) * float(wx)))
    wy2 = F32(-1.0 / (float(wy) * float(wy)))
    ps = F32(pixel_size)
    ps2 = F32(ps * ps)
    flat = out.reshape(-1).copy()
    n = H * nb
    f = np.arange(n)
    j = (f // nb).astype(np.int64)
    i = (f % nb).astype(F32)
    x = (i * ps).astype(F32)
    xw2 = ((x * x).astype(F32) * wx2).astype(F32)
    y2 = (F32(1.0) * (j * j).astype(F32) * ps2).astype(F32)
    yw2 = (y2 * wy2).astype(F32)
    g = np.exp((xw2 + yw2).astype(F32).astype(np.float64)).astype(F32)
    flat[:n] = (flat[:n] * g).astype(F32)
    return flat.reshape(H, Nx)


def snap_tilt(S, kx, ky, k0, aperture_rad, pixel_size):
    """Tilt estimate of one polarisation (digHolo.cpp:11601-11691): DCT-II of
    the batch-summed Fourier intensity S (H, Nx), the Gaussian filter, DCT-III,
    then the maximum over pixels with kx^2 + ky^2 > (2 k0 aperture)^2 (first
    in row-major order on ties); returns (tiltX, tiltY) in degrees and the
    correlation map."""
    H, Nx = S.shape
    out = dct2_redft(np.asarray(S, dtype=F32), 2)
    out = snap_filter(out, k0, aperture_rad, pixel_size)
    out2 = dct2_redft(out, 3)
    aperturek = F32(k0 * F32(aperture_rad))
    ad = F32(aperturek * F32(2))
    ad = F32(ad * ad)
    xs = kx[:Nx].astype(F32)
    ys = ky[:H].astype(F32)
    kr = ((xs * xs)[None, :] + (ys * ys)[:, None]).astype(F32)
    cand = np.where(kr > ad, out2, -np.inf)
    flat = int(np.argmax(cand))          # first maximum in row-major order
    j, i = divmod(flat, Nx)
    tx = F32(F32(np.arcsin(F32(xs[i] / k0))) / UNIT_ANGLE)
    ty = F32(F32(np.arcsin(F32(ys[j] / k0))) / UNIT_ANGLE)
    return tx, ty, out2


def windowed_fourier_aeff(F, kx, ky, cx, cy, radius):
    """Effective area of the batch-summed Fourier intensity inside the disk
    of `radius` around (cx, cy) (digHoloFieldAnalysis with a negative window
    radius, removeZeroOrder1D set: rows 0 and H/2, column 0 and the columns
    from 8 floor(Nx/8) on excluded), intensity |F|^2 / (Nx H)."""
    B, Ny, Nx = F.shape
    xs = kx[:Nx].astype(F32)
    ys = ky[:Ny].astype(F32)
    dx = (xs - F32(cx)).astype(F32)
    dy = (ys - F32(cy)).astype(F32)
    rr = ((dx * dx)[None, :] + (dy * dy)[:, None]).astype(F32)
    w2 = F32(F32(radius) * F32(radius))
    mask = rr <= w2
    nxr = 8 * (Nx // 8)
    mask[:, nxr:] = False
    mask[:, 0] = False
    mask[0, :] = False
    mask[Ny // 2, :] = False
    S = ((np.abs(F) ** 2) * mask[None]).sum(axis=0) / (Nx * Ny)
    P = S.sum()
    E4 = (S ** 2).sum()
    dA = abs(float(kx[2] - kx[1])) * abs(float(ky[2] - ky[1]))
    with np.errstate(invalid="ignore", divide="ignore"):
        return dA * P * P / E4


def aeff_to_mfd(aeff, groups):
    """AeffToMFD (digHolo.cpp:2887-2900)."""
    if not groups:
        return F32(0)
    A = F32(float(aeff) / (15.1059697707643 * groups + 6.65360122093789))
    return F32(2 * float(F32(np.sqrt(F32(A / PI_F)))) / 0.223008930683135)


def focus_estimate(w_camera, w_fourier):
    """FocusEstimate (digHolo.cpp:12017-12050)."""
    if not (w_camera > 0 and w_fourier > 0):
        return F32(0)
    ratio = F32(F32(w_fourier) / F32(w_camera))
    a, b = F32(0.25), F32(PI_F / F32(2))
    with np.errstate(invalid="ignore"):
        r = F32(F32(2) * F32(b * F32(np.sqrt(F32(F32(F32(1) - a) / F32(ratio - a)) - F32(1)))))
    if not (r > 0) or np.isnan(r):
        return F32(0)
    return r


def fit_quadratic(x, y, B0, tol=1e-6, max_iter=1000):
    """fitToQuadratic (digHolo.cpp:3146-3255): Gauss-Newton steps of
    y = a x^2 + b x + c solved by least squares; the residual accumulates
    over the iterations as in the reference.  Returns (x of the extremum,
    B)."""
    a, b, c = (F32(v) for v in B0)
    x = np.asarray(x, dtype=F32)
    y = np.asarray(y, dtype=F32)
    resid = F32(0)
    last = F32(0)
    it = 0
    B = [a, b, c]
    while True:
        J = np.stack([(x * x).astype(F32), x, np.ones_like(x)], axis=1)
        r = (y - ((a * x * x).astype(F32) + (b * x).astype(F32) + c).astype(F32)).astype(F32)
        if np.isnan(J).any() or np.isnan(r).any():
            return float("nan"), B
        resid = F32(resid + F32((r.astype(F32) * r.astype(F32)).sum(dtype=F32)))
        d = np.linalg.lstsq(J.astype(np.float64), r.astype(np.float64), rcond=None)[0].astype(F32)
        a, b, c = F32(a + d[0]), F32(b + d[1]), F32(c + d[2])
        B = [a, b, c]
        it += 1
        done = abs(float(resid - last)) < tol or it > max_iter
        last = resid
        mx = F32(-b / F32(2 * a))
        if done:
            return float(mx), B


def _untilted_fields(frames, cfg):
    res = process_batch(frames, _no_basis(cfg), quantised=True)
    return res


def _no_basis(cfg):
    import copy
    c = copy.deepcopy(cfg)
    c.max_mg = 0
    return c


def auto_focus(res, cfg, scale):
    """digHoloAutoFocus (digHolo.cpp:11181-11499): per defocus trial, the
    tilt-removed field V = -conj(A . ref) (float, before int16 rounding) is
    transformed back (unnormalised backward DFT of the field plane) and the
    effective area of its batch-summed intensity scored; up to 25 trials,
    the first two at +-scale, then a 0.25-scale ladder from the better one,
    from the fifth on the minimum of a quadratic fitted to the four smallest
    effective areas.  Returns the defocus with the smallest effective area
    per polarisation."""
    import copy
    P = cfg.pol_count
    W, H = res["W"], res["H"]
    kx, ky = res["kx"], res["ky"]
    xax, yax = res["x"], res["y"]
    dA = F32(abs(float(kx[2] - kx[1])) * abs(float(ky[2] - ky[1])))
    E = res["field_untilted"]
    step_count, fit_count = 25, 5
    scale = [max(F32(s), F32(1.0)) for s in scale]
    defoc = np.zeros((P, step_count + 3), dtype=F32)
    aeffs = np.zeros((P, step_count + 3), dtype=F32)
    s0 = list(scale)
    for st in range(0, step_count, 2):
        for p in range(P):
            defoc[p, st] = s0[p]
            defoc[p, st + 1] = -s0[p]
            s0[p] = F32(s0[p] + F32(scale[p] * F32(0.25)))
    best_aeff = [np.inf] * P
    best = [F32(0)] * P
    converged = [False] * P
    B0 = [[F32(0)] * 3 for _ in range(P)]
    Bf = [[F32(0)] * 3 for _ in range(P)]
    for st in range(step_count):
        c = copy.deepcopy(cfg)
        for p in range(P):
            c.defocus[p] = F32(defoc[p, st])
        total = True
        for p in range(P):
            refx, refy = reference_wave(c, p, xax, yax, W, H, res["SX"], res["SY"], kx[1] - kx[0], ky[1] - ky[0], True)
            V, _, _ = apply_tilt(E[:, p], refx, refy, np.ones(E.shape[0]), True)
            V = V.astype(np.complex64)
            Fo = np.fft.ifft2(V) * (V.shape[-1] * V.shape[-2])
            S = (np.abs(Fo) ** 2).sum(axis=0)
            v2 = float(S.sum())
            v4 = float((S ** 2).sum())
            a = F32(float(dA) * (v2 * v2) / v4)
            aeffs[p, st] = a
            if a < best_aeff[p]:
                best_aeff[p] = a
                best[p] = F32(defoc[p, st])
            if st == 1:
                if aeffs[p, 1] < aeffs[p, 0]:
                    sc, base = F32(defoc[p, 1] - defoc[p, 0]), defoc[p, 1]
                else:
                    sc, base = F32(defoc[p, 0] - defoc[p, 1]), defoc[p, 0]
                idx = 1
                for i in range(2, step_count, 2):
                    defoc[p, i] = F32(base + F32(F32(idx * 0.25) * sc))
                    defoc[p, i + 1] = F32(base - F32(F32(idx * 0.25) * sc))
                    idx += 1
            if st >= fit_count - 1:
                if st == fit_count - 1:
                    B0[p] = [F32(1e7), F32(1e7), F32(sum(float(aeffs[p, i]) for i in range(st)) / (st + 1))]
                xs = defoc[p, :st + 1].copy()
                ys = aeffs[p, :st + 1].copy()
                # sortIt (digHolo.cpp:11161-11179): ascending effective area, stable
                order = np.argsort(ys, kind="stable")
                xs, ys = xs[order], ys[order]
                mx, Bf[p] = fit_quadratic(xs[:fit_count - 1], ys[:fit_count - 1], B0[p])
                B0[p] = list(Bf[p])
                if st + 1 < step_count - 1:
                    if not np.isnan(mx):
                        defoc[p, st + 1] = F32(mx)
                if abs(mx - float(best[p])) < 0.01:
                    converged[p] = True
            total = total and converged[p]
        if total:
            break
    return best


def auto_align_snap(frames, cfg, align_tilt=1, align_defocus=1, align_centre=1, align_waist=1,
                    align_radius=1, pols_independent=0):
    """digHoloAutoAlignSnap (digHolo.cpp:11517-11970) with the aperture rule
    AutoAlign applies before it (digHolo.cpp:12286-12299).  Returns the
    estimated configuration (a new Config) and the search step sizes."""
    import copy
    c = copy.deepcopy(cfg)
    P = c.pol_count
    fw, fh = c.frame_width, c.frame_height
    ps = F32(c.pixel_size)
    lam = F32(c.wavelength)
    if align_radius:
        if align_tilt:
            wc = (-2.0 + math.sqrt(68.0)) / 16.0
            wmax = F32(float(lam) / (2.0 * float(ps)))
            c.window_radius_deg = F32(F32(F32(wc) * wmax) / UNIT_ANGLE)
        else:
            c.window_radius_deg = F32(min(F32(np.sqrt(F32(F32(t[0] * t[0]) + F32(t[1] * t[1])))) for t in c.tilt_deg[:P]) / F32(3))
    for p in range(P):
        if align_centre:
            c.beam_centre[p] = [F32((-(P - 1) * (fw / 4.0) + (p * fw / 2.0)) * float(ps)), F32(0)]
        if align_tilt:
            c.tilt_deg[p] = [F32(0), F32(0)]
        if align_defocus:
            c.defocus[p] = F32(0)
    c.fft_window = (fw // P, fh)
    W, H, cxs, cys = fft_windows(c)
    kx, ky = k_axes(W, H, ps)
    Fp = r2c_windows(frames, c, W, H, cxs, cys)
    k0 = F32(F32(2) * PI_F / lam)
    fa = [fourier_analysis(Fp[:, p], kx, ky, lam, c.window_radius_deg) for p in range(P)]
    waistF = [F32(0)] * P
    tilts = {}
    for pas in range(1 + (1 if align_radius else 0)):
        for p in range(P):
            ap = F32(c.window_radius_deg * UNIT_ANGLE)
            tx, ty, _ = snap_tilt(fa[p]["batchsum"].astype(F32), kx, ky, k0, ap, ps)
            tilts[(pas, p)] = (tx, ty)
            if align_radius:
                apmax = F32(F32(np.sqrt(F32(F32(tx * tx) + F32(ty * ty)))) / F32(3))
                if apmax < c.window_radius_deg:
                    c.window_radius_deg = apmax
                    fa = [fourier_analysis(Fp[:, q], kx, ky, lam, c.window_radius_deg) for q in range(P)]
            if align_tilt:
                c.tilt_deg[p] = [tx, ty]
            wcx = F32(k0 * F32(c.tilt_deg[p][0] * UNIT_ANGLE))
            wcy = F32(k0 * F32(c.tilt_deg[p][1] * UNIT_ANGLE))
            wr = F32(k0 * F32(np.sin(F32(c.window_radius_deg * UNIT_ANGLE))))
            aeff = windowed_fourier_aeff(Fp[:, p], kx, ky, wcx, wcy, wr)
            west = aeff_to_mfd(aeff, c.max_mg)
            waistF[p] = F32(PI_F / west) if west else F32(np.inf)
    # camera plane (digHolo.cpp:11791-11902)
    max_focus = F32(0.25)
    est = [F32(0)] * P
    attempts = 0
    valid = False
    res = None
    while (not valid or attempts == 0) and attempts < 10:
        valid = True
        res = _untilted_fields(frames, c)
        B = res["field_untilted"].shape[0]
        for p in range(P):
            off = F32(((2 * p - 1) * float(ps) * fw / 4.0) * (P - 1))
            st = res["stats"][p]
            comx = F32(F32(st["comx"][B]) + off)
            comy = F32(st["comy"][B])
            aeff = F32(st["aeff"][B])
            west = F32(aeff_to_mfd(aeff, c.max_mg) * F32(0.5))
            est[p] = focus_estimate(west, waistF[p])
            if np.isnan(comx) or np.isnan(comy) or np.isnan(aeff):
                valid = False
                c.window_radius_deg = F32(c.window_radius_deg * F32(0.9))
            if valid:
                if align_centre:
                    c.beam_centre[p] = [comx, comy]
                if align_waist:
                    c.waist[p] = west
                if align_defocus:
                    c.defocus[p] = F32(0)
                max_focus = max(max_focus, abs(est[p]))
            attempts += 1
    if align_defocus:
        # the fields of the last camera-plane pass: the Fourier planes of the
        # windows placed at the reset centres, the beam-centre phase of that pass
        best = auto_focus(res, c, est)
        for p in range(P):
            c.defocus[p] = best[p]
            max_focus = max(max_focus, abs(best[p]))
    steps = {"tilt": F32(c.window_radius_deg * F32(0.1)), "centre": F32(c.waist[0] * F32(0.1)),
             "defocus": F32(F32(0.1) * max_focus), "waist": F32(c.waist[0] * F32(0.1))}
    c.fft_window = cfg.fft_window
    return c, steps, {"tilts": tilts, "waist_fourier": waistF, "focus_estimate": est}


def frame_simulator(frame_count, frame_width, frame_height, pixel_size, pol_count, ref_tilt_x=None, ref_tilt_y=None,
                    ref_defocus=None, ref_waist=None, ref_centre_x=None, ref_centre_y=None, group_count=0,
                    beam_waist=None, beam_coefs=None, beam_centre_x=None, beam_centre_y=None, levels=16384,
                    fill_factor=1, wavelengths=None):
    """frameSimulatorCreate (digHolo.cpp:15930-16760) for small cases: the
    frames (float32, quantised, and uint16) and the resolved parameters.

    The reference's region axes are transposed against its frame layout: its
    x axis (beam centre x, reference tilt x, HG index n) runs along the
    frame's rows and its y axis along a polarisation region's columns
    (digHolo.cpp:16371-16385 with generateModeSeparable's transpose,
    digHolo.cpp:1610-1760).  The field is accumulated in the reference's
    float32 order: first mode's term plus the reference wave, then every later
    mode with nonzero coefficient power and the last mode; the fill-factor
    sinc filter is applied in FP64 (FFTW's single-precision rounding differs
    in the last bits); quantisation against the pre-filter maximum with
    round-half-even (digHolo.cpp:15847-15873).  With no group count and a
    frame count that is not triangular, the one-hot default coefficients use
    the final mode count (the reference reads memory it never wrote there).
    """
    W = 16 * (frame_width // 16)
    H = 16 * (frame_height // 16)
    P = min(pol_count, 2)
    ps = F32(pixel_size if pixel_size > 0 else 20e-6)
    if levels < 2 or levels > 65536:
        levels = 65536
    G = group_count
    if G <= 0:
        m, g = 0, 1
        while m < frame_count:
            m += g
            g += 1
        G = g - 1 if m == frame_count else g
    M = G * (G + 1) // 2
    wl = [F32(1565e-9)] if wavelengths is None else [F32(v) for v in wavelengths]
    k0 = F32(0)
    for v in wl:
        k0 = F32(k0 + F32(F32(2 * PI_F) / v))
    k0 = F32(k0 / F32(len(wl)))
    lam0 = F32(F32(2 * PI_F) / k0)
    wmax = F32(lam0 / F32(2 * ps))
    unit = F32(PI_F / F32(180))
    tilt_max = F32(float(wmax) * (1 - 0.32037724101704079249230971981887705624103546142578125) / float(unit))
    rows, cols = H, W // P
    off = [F32((float(ps) * (W // P) / 2.0) * (P * p - (P - 1))) for p in range(P)]
    pick = lambda arr, p, d: F32(arr[p]) if arr is not None else F32(d)
    tx = [pick(ref_tilt_x, p, tilt_max) for p in range(P)]
    ty = [pick(ref_tilt_y, p, -tilt_max) for p in range(P)]
    df = [pick(ref_defocus, p, 0) for p in range(P)]
    rw = [pick(ref_waist, p, 0) for p in range(P)]
    rcx = [pick(ref_centre_x, p, off[p]) for p in range(P)]
    rcy = [pick(ref_centre_y, p, 0) for p in range(P)]
    bcx = [pick(beam_centre_x, p, off[p]) for p in range(P)]
    bcy = [pick(beam_centre_y, p, 0) for p in range(P)]
    if beam_waist is None:
        r = F32(0.25 * min(rows, cols) * float(ps))
        w = F32(aeff_to_mfd(F32(PI_F * r * r), G) * F32(0.5))
        bw = [w] * P
    else:
        bw = [F32(v) for v in beam_waist]
    if beam_coefs is None:
        coefs = np.zeros((frame_count, P, M), dtype=np.complex64)
        for f in range(min(frame_count, M)):
            coefs[f, :, f] = 1
    else:
        coefs = np.asarray(beam_coefs, dtype=np.complex64).reshape(frame_count, P, M)
    idx = hg_index(G)
    out = np.zeros((frame_count, H, W), dtype=F32)
    vmax = F32(0)
    for p in range(P):
        ax_r = (ps * (np.arange(rows) - rows // 2).astype(F32) + F32(off[p] - bcx[p])).astype(F32)
        ax_c = (ps * (np.arange(cols) - cols // 2).astype(F32) + F32(-bcy[p])).astype(F32)
        qr, sr = quantise_modes(hg_modes(ax_r, bw[p], G))
        qc, sc = quantise_modes(hg_modes(ax_c, bw[p], G))
        ref = []
        for ax_len, ctr, kt, axis_idx in ((rows, rcx[p], tx[p], 0), (cols, rcy[p], ty[p], 1)):
            shift = F32(off[p] - ctr) if axis_idx == 0 else F32(-ctr)
            a = (ps * (np.arange(ax_len) - ax_len // 2).astype(F32) + shift).astype(F32)
            kr = F32(k0 * F32(np.sin(F32(kt * unit))))
            kf = F32(k0 * F32(F32(0.5) * df[p]))
            r2 = (a * a).astype(F32)
            arg = (kr * a + kf * r2).astype(F32)
            A0 = F32(np.sqrt(F32(1.0) / F32(ax_len)))
            A = (A0 * np.exp(-r2 / F32(rw[p] * rw[p]))).astype(F32) if rw[p] * rw[p] > 0 else np.full(ax_len, A0, F32)
            ref.append(((A * np.cos(arg)).astype(F32), (A * np.sin(arg)).astype(F32)))
        (rrr, rri), (rcr, rci) = ref
        # cmul(column factor, row factor) with the real part fused
        ref_re = (rcr[None, :].astype(np.float64) * rrr[:, None] - (rci[None, :] * rri[:, None]).astype(F32)).astype(F32)
        ref_im = (rcr[None, :].astype(np.float64) * rri[:, None] + (rci[None, :] * rrr[:, None]).astype(F32)).astype(F32)
        for f in range(frame_count):
            fr = fi = None
            for k, (m, n) in enumerate(idx):
                c = coefs[f, p, k]
                cR = F32(float(sc[m]) * float(sr[n]) * float(c.real))
                cI = F32(float(sc[m]) * float(sr[n]) * float(c.imag))
                if not (F32(cR * cR + cI * cI) > 0 or k == 0 or k == M - 1):
                    continue
                v = (qr[n].astype(np.int32)[:, None] * qc[m].astype(np.int32)[None, :]).astype(F32)
                tr, ti = (v * cR).astype(F32), (v * cI).astype(F32)
                if fr is None:
                    fr, fi = (ref_re + tr).astype(F32), (ref_im + ti).astype(F32)
                else:
                    fr, fi = (tr + fr).astype(F32), (ti + fi).astype(F32)
            I = ((fr * fr).astype(F32) + (fi * fi).astype(F32)).astype(F32)
            out[f, :, p * cols:(p + 1) * cols] = I
            vmax = max(vmax, F32(I.max()))
    if fill_factor:
        period = F32(2.0 * float(ps))
        kfx = F32(2 * (2.0 * math.pi / float(period)) / W)
        kfy = F32(2 * (2.0 * math.pi / float(period)) / H)
        kx = (kfx * np.array([i if i <= W // 2 else i - W for i in range(W // 2 + 1)], dtype=F32)).astype(F32)
        ky = (kfy * np.array([i if i <= H // 2 else i - H for i in range(H)], dtype=F32)).astype(F32)
        with np.errstate(invalid="ignore", divide="ignore"):
            ax = (kx * F32(0.5) * ps).astype(F32)
            ay = (ky * F32(0.5) * ps).astype(F32)
            sx = np.where(kx != 0, np.sin(ax) / ax, 1).astype(F32)
            sy = np.where(ky != 0, np.sin(ay) / ay, 1).astype(F32)
        env = ((sy * F32(1.0 / (W * H))).astype(F32)[:, None] * sx[None, :]).astype(F32)
        for f in range(frame_count):
            X = np.fft.rfft2(out[f].astype(np.float64)) * env
            out[f] = np.fft.irfft2(X, s=(H, W)) * (W * H)
    inv = F32(F32(levels - 1) / vmax)
    q = np.rint((out * inv).astype(F32)).astype(F32)
    q16 = np.clip(q, 0, 65535).astype(np.uint16)
    params = dict(W=W, H=H, P=P, G=G, M=M, tilt_x=tx, tilt_y=ty, beam_waist=bw, beam_centre_x=bcx,
                  ref_centre_x=rcx, coefs=coefs, levels=levels, pixel_size=ps)
    return q, q16, params
