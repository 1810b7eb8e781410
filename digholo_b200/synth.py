"""Seeded synthetic off-axis holograms with the shapes of the benchmark workloads.

There is no public dataset behind the digHolo benchmarks; every input is
generated here.  The model (one polarisation region of a camera frame):

    I = |R + S|^2 + N
    R = exp(i (kx x + ky y)),  |R| = 1,  (kx, ky) = carrier * (pi / pixelSize)
    S = sum_mn c_mn HG_m(x - x0) HG_n(y - y0),  sum |S|^2 = signalFraction * sum |R|^2
    N ~ Normal(0, sigma^2),  sigma = mean(|R+S|^2) * 10^(-SNR/20)

HG_m is the unit-power Hermite-Gaussian of waist w0, evaluated in FP64 by the
normalised three-term recurrence.  Dual-polarisation frames hold polarisation
0 in the left half and polarisation 1 in the right half (beam centres at
-+ frameWidth/4 pixels from the frame centre), each half with its own carrier.
uint16 frames are scaled so the batch maximum of the clean intensity maps to
4095, noise is added, and the result is rounded and clipped to 0..4095
(12-bit camera).

The tilt to give digHolo for a carrier c (in Nyquist units) is
``carrier_to_tilt_degrees``: the reference removes the carrier with the
small-angle phase -k0*theta*x (digHolo.cpp:10440-10441), so theta = kx/k0.
"""
import math

import numpy as np

WAVELENGTH = 1565e-9
PIXEL_SIZE = 20e-6


def hg_modes_1d(u_axis, w0, count):
    """Unit-power HG modes (count x len(axis)) sampled on ``u_axis`` (metres).

    Normalised so that sum_x HG_m(x)^2 * dx == 1 in the continuum limit,
    i.e. HG_m(x) = (2/pi)^(1/4) / sqrt(w0) * psi_m(sqrt(2) x / w0) with
    psi_m the normalised Hermite function.
    """
    u = np.sqrt(2.0) * np.asarray(u_axis, dtype=np.float64) / w0
    out = np.zeros((count, u.size), dtype=np.float64)
    g = np.exp(-0.5 * u * u) * math.pi ** -0.25
    out[0] = g
    if count > 1:
        out[1] = math.sqrt(2.0) * u * g
    for n in range(2, count):
        out[n] = math.sqrt(2.0 / n) * u * out[n - 1] - math.sqrt((n - 1.0) / n) * out[n - 2]
    return out * (2.0 ** 0.25) / math.sqrt(w0)


def hg_indices(max_mg):
    """(m, n) pairs in digHolo's order: group g, then (g-k, k) for k = 0..g (digHolo.cpp:1245-1265)."""
    ms, ns = [], []
    for g in range(max(max_mg, 1)):
        for k in range(g + 1):
            ms.append(g - k)
            ns.append(k)
    return np.array(ms), np.array(ns)


def carrier_to_tilt_degrees(carrier, pixel_size=PIXEL_SIZE, wavelength=WAVELENGTH):
    k0 = 2 * math.pi / wavelength
    return math.degrees((carrier * math.pi / pixel_size) / k0)


def window_radius_degrees(carrier_xy, pixel_size=PIXEL_SIZE, wavelength=WAVELENGTH):
    """Fourier window radius = |tilt| / 3, the reference's own rule (digHolo.cpp:11973-11976)."""
    tx = carrier_to_tilt_degrees(carrier_xy[0], pixel_size, wavelength)
    ty = carrier_to_tilt_degrees(carrier_xy[1], pixel_size, wavelength)
    return math.hypot(tx, ty) / 3.0


class Hologram:
    """A generated batch plus the settings that reconstruct it."""

    def __init__(self, frames, pol_count, frame_width, frame_height, beam_centres, tilts_deg,
                 waist, max_mg, coefs, window, radius_deg, pixel_size, wavelength):
        self.frames = frames
        self.pol_count = pol_count
        self.frame_width = frame_width
        self.frame_height = frame_height
        self.beam_centres = beam_centres
        self.tilts_deg = tilts_deg
        self.waist = waist
        self.max_mg = max_mg
        self.coefs = coefs
        self.window = window
        self.radius_deg = radius_deg
        self.pixel_size = pixel_size
        self.wavelength = wavelength


def transfer_coefs(frame_count, pol_count, max_mg, seed, loss_db=1.0):
    """Coefficients of frames that each excite one column of a Haar-random
    unitary over the modes of all polarisations (pol_count * M square),
    times a per-mode loss uniform in [0, loss_db] dB: frame f carries column
    f mod (pol_count * M) of diag(d) U, whose rows split into the
    polarisations (rows p M .. p M + M - 1 are polarisation p).  The batch
    coefficient matrix of both polarisations together then has full rank
    once frame_count >= pol_count * M."""
    rng = np.random.default_rng(seed)
    M = len(hg_indices(max_mg)[0])
    N = pol_count * M
    z = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))[None, :]   # Haar: fix the phases of R's diagonal
    d = 10.0 ** (-rng.uniform(0.0, loss_db, size=N) / 20.0)
    T = d[:, None] * q
    out = np.zeros((frame_count, pol_count, M), dtype=np.complex128)
    for f in range(frame_count):
        out[f] = T[:, f % N].reshape(pol_count, M)
    return out


def generate(frame_count, frame_width, frame_height, pol_count, max_mg, waist, snr_db,
             carrier=(0.25, 0.2), window=(64, 64), dtype="float32", seed=1000,
             centre_jitter=40e-6, signal_fraction=0.1, taper=False, coefs=None,
             pixel_size=PIXEL_SIZE, wavelength=WAVELENGTH, defocus=0.0, normalise_frames=True):
    """Generate ``frame_count`` frames (frame_count, frame_height, frame_width).

    ``coefs`` may be given as (frame_count, pol_count, modeCount) complex; by
    default they are i.i.d. complex Gaussian, optionally tapered by
    1/(group+1).  Returns a :class:`Hologram`.
    """
    rng = np.random.default_rng(seed)
    ms, ns = hg_indices(max_mg)
    mode_count = ms.size
    region_w = frame_width // pol_count
    xs = (np.arange(frame_width) - frame_width // 2) * pixel_size
    ys = (np.arange(frame_height) - frame_height // 2) * pixel_size
    nyq = math.pi / pixel_size

    centres = []
    carriers = []
    for pol in range(pol_count):
        base_x = 0.0 if pol_count == 1 else (-frame_width / 4.0 if pol == 0 else frame_width / 4.0) * pixel_size
        off = rng.uniform(-centre_jitter, centre_jitter, size=2)
        centres.append((base_x + off[0], off[1]))
        sgn = 1.0 if pol == 0 else -1.0
        carriers.append((sgn * carrier[0], sgn * carrier[1]))

    if coefs is None:
        coefs = (rng.standard_normal((frame_count, pol_count, mode_count)) +
                 1j * rng.standard_normal((frame_count, pol_count, mode_count))) / math.sqrt(2.0)
        if taper:
            coefs = coefs / (ms + ns + 1.0)[None, None, :]
    coefs = np.asarray(coefs, dtype=np.complex128)

    clean = np.zeros((frame_count, frame_height, frame_width), dtype=np.float64)
    for pol in range(pol_count):
        x0 = pol * region_w
        xr = xs[x0:x0 + region_w]
        cx, cy = centres[pol]
        hx = hg_modes_1d(xr - cx, waist, max_mg)          # (G, region_w)
        hy = hg_modes_1d(ys - cy, waist, max_mg)          # (G, H)
        kx, ky = carriers[pol][0] * nyq, carriers[pol][1] * nyq
        ref = np.exp(1j * ky * ys)[:, None] * np.exp(1j * kx * xr)[None, :]   # (H, region_w)
        npix = ref.size
        for f0 in range(0, frame_count, 64):
            f1 = min(frame_count, f0 + 64)
            cmat = np.zeros((f1 - f0, max_mg, max_mg), dtype=np.complex128)
            cmat[:, ms, ns] = coefs[f0:f1, pol, :]
            # S[f, y, x] = sum_mn c_mn hy[n, y] hx[m, x]
            s = np.einsum("fmn,ny,mx->fyx", cmat, hy, hx, optimize=True)
            if defocus:
                # quadratic phase of a defocus of `defocus` dioptres about the beam centre
                r2 = ((ys - cy) ** 2)[:, None] + ((xr - cx) ** 2)[None, :]
                s = s * np.exp(1j * math.pi * defocus * r2 / wavelength)[None]
            if normalise_frames:
                p = np.sum(np.abs(s) ** 2, axis=(1, 2), keepdims=True)
                s = s * np.sqrt(signal_fraction * npix / np.maximum(p, 1e-300))
            else:
                # one scale for the whole batch, so relative frame powers (mode-dependent loss)
                # survive: sum over pixels of |S|^2 ~ sum |c|^2 / pixel^2 for unit-power HG modes
                mean_c2 = float(np.mean(np.sum(np.abs(coefs[:, pol, :]) ** 2, axis=1)))
                s = s * math.sqrt(signal_fraction * npix * pixel_size ** 2 / max(mean_c2, 1e-300))
            clean[f0:f1, :, x0:x0 + region_w] = np.abs(ref[None] + s) ** 2

    sigma = clean.mean() * 10.0 ** (-snr_db / 20.0)
    noise = rng.standard_normal(clean.shape) * sigma
    if dtype == "uint16":
        scale = 4095.0 / clean.max()
        frames = np.clip(np.rint((clean + noise) * scale), 0, 4095).astype(np.uint16)
    else:
        frames = (clean + noise).astype(np.float32)

    # digHolo reconstructs only from kx >= 0 (digHolo.cpp:8002-8007), so every
    # polarisation is configured with the positive carrier: for a negative
    # carrier that window holds the conjugate twin term R* S.
    tilts = [(carrier_to_tilt_degrees(abs(c[0]), pixel_size, wavelength),
              carrier_to_tilt_degrees(abs(c[1]), pixel_size, wavelength)) for c in carriers]
    radius = window_radius_degrees(carrier, pixel_size, wavelength)
    return Hologram(frames, pol_count, frame_width, frame_height, centres, tilts, waist, max_mg,
                    coefs, window, radius, pixel_size, wavelength)


# Workload shapes (frame counts can be reduced for parity tests).
WORKLOADS = {
    "plain_320x256_f32_1pol": dict(frame_count=16, frame_width=320, frame_height=256, pol_count=1,
                                   max_mg=9, waist=200e-6, snr_db=30, window=(64, 64),
                                   dtype="float32", seed=1001),
    "batched_640x512_u16_2pol": dict(frame_count=1024, frame_width=640, frame_height=512, pol_count=2,
                                     max_mg=15, waist=250e-6, snr_db=25, window=(128, 128),
                                     dtype="uint16", seed=1002),
    # frames excite columns of a Haar-random 120x120 transfer matrix with per-mode loss
    # (coefficients from transfer_coefs); frames are not normalised individually
    # carrier (0.55, 0.45) of Nyquist: the Fourier window (radius |tilt| / 3)
    # then holds all 120 modes of each polarisation at this waist (with the
    # (0.25, 0.2) carrier the higher mode groups fall outside it and the batch
    # coefficient matrix loses rank)
    "align_640x512_f32_2pol": dict(frame_count=512, frame_width=640, frame_height=512, pol_count=2,
                                   max_mg=15, waist=250e-6, snr_db=30, window=(128, 128),
                                   carrier=(0.55, 0.45), dtype="float32", seed=1004, normalise_frames=False),
    # the same frames with the (0.25, 0.2) carrier: the parameter-estimate
    # (snap) tests, whose parity with the reference was established on them
    "snap_640x512_f32_2pol": dict(frame_count=512, frame_width=640, frame_height=512, pol_count=2,
                                  max_mg=15, waist=250e-6, snr_db=30, window=(128, 128),
                                  dtype="float32", seed=1004, normalise_frames=False),
    "largefield_2048_u16_2pol": dict(frame_count=256, frame_width=2048, frame_height=2048, pol_count=2,
                                     max_mg=30, waist=600e-6, snr_db=20, window=(512, 512),
                                     dtype="uint16", seed=1005, taper=True),
}
