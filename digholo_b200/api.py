"""Helpers that drive any library exposing the digHolo C ABI (this
project's libdigholo_b200.so, or the reference build) from numpy: apply a
configuration through the setters, run a batch, and copy the outputs."""
import ctypes as C

import numpy as np


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def configure(L, h, cfg):
    """Apply a configuration object through the ConfigSet* entry points.

    ``cfg`` needs: frame_width, frame_height, pixel_size, wavelength,
    pol_count, fft_window, window_radius_deg, resolution_mode, max_mg,
    fill_factor, pol_lock_tilt, pol_lock_defocus, pol_lock_waist, and
    per-polarisation waist, beam_centre, tilt_deg, defocus; optionally
    batch_cal, complex (polCount, batchCount) batch calibration factors;
    basis_type (0 HG, 1 LG, 2 custom with basis_custom, complex [in][out]).
    """
    L.digHoloConfigSetFrameDimensions(h, int(cfg.frame_width), int(cfg.frame_height))
    L.digHoloConfigSetFramePixelSize(h, float(cfg.pixel_size))
    L.digHoloConfigSetWavelengthCentre(h, float(cfg.wavelength))
    L.digHoloConfigSetPolCount(h, int(cfg.pol_count))
    L.digHoloConfigSetfftWindowSize(h, int(cfg.fft_window[0]), int(cfg.fft_window[1]))
    L.digHoloConfigSetFourierWindowRadius(h, float(cfg.window_radius_deg))
    L.digHoloConfigSetIFFTResolutionMode(h, int(cfg.resolution_mode))
    L.digHoloConfigSetBasisGroupCount(h, int(cfg.max_mg))
    L.digHoloConfigSetFillFactorCorrectionEnabled(h, int(cfg.fill_factor))
    L.digHoloConfigSetPolLockTilt(h, int(cfg.pol_lock_tilt))
    L.digHoloConfigSetPolLockDefocus(h, int(cfg.pol_lock_defocus))
    L.digHoloConfigSetPolLockBasisWaist(h, int(cfg.pol_lock_waist))
    for p in range(int(cfg.pol_count)):
        L.digHoloConfigSetBasisWaist(h, p, float(cfg.waist[p]))
        L.digHoloConfigSetBeamCentre(h, 0, p, float(cfg.beam_centre[p][0]))
        L.digHoloConfigSetBeamCentre(h, 1, p, float(cfg.beam_centre[p][1]))
        L.digHoloConfigSetTilt(h, 0, p, float(cfg.tilt_deg[p][0]))
        L.digHoloConfigSetTilt(h, 1, p, float(cfg.tilt_deg[p][1]))
        L.digHoloConfigSetDefocus(h, p, float(cfg.defocus[p]))
    bt = int(getattr(cfg, "basis_type", 0) or 0)
    if bt == 1:
        L.digHoloConfigSetBasisTypeLG(h)
    elif bt == 2:
        t = np.ascontiguousarray(np.asarray(cfg.basis_custom, dtype=np.complex64))
        L.digHoloConfigSetBasisTypeCustom(h, t.shape[0], t.shape[1], t.ctypes.data_as(C.POINTER(C.c_float)))
    else:
        L.digHoloConfigSetBasisTypeHG(h)
    cal = getattr(cfg, "batch_cal", None)
    if cal is not None:
        c = np.ascontiguousarray(np.asarray(cal, dtype=np.complex64))
        L.digHoloConfigSetBatchCalibration(h, c.ctypes.data_as(C.POINTER(C.c_float)), c.shape[0], c.shape[1])


def set_batch(L, h, frames):
    """digHoloSetBatch / digHoloSetBatchUint16 on a contiguous numpy batch.
    The array must stay alive until processing is done (the library keeps
    only the pointer, as the reference does)."""
    B = frames.shape[0]
    if frames.dtype == np.uint16:
        return L.digHoloSetBatchUint16(h, B, ptr(frames, C.c_ushort), 0)
    return L.digHoloSetBatch(h, B, ptr(frames, C.c_float))


def set_batch_avg(L, h, frames, avg_count, avg_mode):
    """digHoloSetBatchAvg / digHoloSetBatchAvgUint16: frames holds batchCount *
    avg_count frames, averaged in groups of avg_count (avg_mode 0: adjacent
    frames, 1: interlaced, 2: sweeps)."""
    B = frames.shape[0] // avg_count
    if frames.dtype == np.uint16:
        return L.digHoloSetBatchAvgUint16(h, B, ptr(frames, C.c_ushort), avg_count, avg_mode, 0)
    return L.digHoloSetBatchAvg(h, B, ptr(frames, C.c_float), avg_count, avg_mode)


def read_outputs(L, h, B, coef_ptr=None, m=0, pc=0, want_fields=True):
    """Copy coefficients, int16 fields, complex fields and the plane-1 summary."""
    out = {}
    if coef_ptr and m > 0:
        arr = np.ctypeslib.as_array(coef_ptr, shape=(B * pc * m * 2,)).copy()
        out["coefs"] = arr.view(np.complex64).reshape(B, pc, m)
    else:
        out["coefs"] = None
    if not want_fields:
        return out
    b, p = C.c_int(), C.c_int()
    fr, fi = C.POINTER(C.c_short)(), C.POINTER(C.c_short)()
    fs = C.POINTER(C.c_float)()
    x, y = C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    w, hh = C.c_int(), C.c_int()
    L.digHoloGetFields16(h, C.byref(b), C.byref(p), C.byref(fr), C.byref(fi), C.byref(fs),
                         C.byref(x), C.byref(y), C.byref(w), C.byref(hh))
    n = b.value * p.value * w.value * hh.value
    shape = (b.value, p.value, hh.value, w.value)
    out["R"] = np.ctypeslib.as_array(fr, shape=(n,)).copy().reshape(shape)
    out["I"] = np.ctypeslib.as_array(fi, shape=(n,)).copy().reshape(shape)
    out["x"] = np.ctypeslib.as_array(x, shape=(w.value,)).copy()
    out["y"] = np.ctypeslib.as_array(y, shape=(hh.value,)).copy()
    fp = L.digHoloGetFields(h, C.byref(b), C.byref(p), C.byref(x), C.byref(y), C.byref(w), C.byref(hh))
    out["field"] = np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64).reshape(shape)
    pcount, tcount, pcn = C.c_int(), C.c_int(), C.c_int()
    params = C.POINTER(C.c_float)()
    px, py = C.c_int(), C.c_int()
    xa, ya, ti = C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    rc = L.digHoloBatchGetSummary(h, 1, C.byref(pcount), C.byref(tcount), C.byref(pcn), C.byref(params),
                                  C.byref(px), C.byref(py), C.byref(xa), C.byref(ya), C.byref(ti))
    if rc == 0:
        stats = np.ctypeslib.as_array(params, shape=(pcount.value * pcn.value * tcount.value,)).copy()
        out["summary"] = stats.reshape(pcount.value, pcn.value, tcount.value)
        out["scale"] = out["summary"][3, :, :B]
        # per polarisation the plane occupies the first nx ny of W H floats (the
        # reference sizes every batch-sum plane by the FFT window)
        W = L.digHoloConfigGetfftWindowSizeX(h)
        Hh = L.digHoloConfigGetfftWindowSizeY(h)
        stride = max(W * Hh, px.value * py.value)
        tot = np.ctypeslib.as_array(ti, shape=(pcn.value * stride,)).copy().reshape(pcn.value, stride)
        out["batch_intensity"] = tot[:, :px.value * py.value].reshape(pcn.value, py.value, px.value)
    return out


def run_batch(L, h, frames, want_fields=True):
    """SetBatch + ProcessBatch + read_outputs on a numpy batch."""
    frames = np.ascontiguousarray(frames)
    if frames.dtype != np.uint16:
        frames = frames.astype(np.float32, copy=False)
    set_batch(L, h, frames)
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    return read_outputs(L, h, frames.shape[0], cp, m.value, pc.value, want_fields)


def read_fourier(L, h):
    """digHoloGetFourierPlaneFull and the plane-0 (Fourier plane) summary of
    digHoloBatchGetSummary.  The plane is returned as (batch, pol, H, W/2+1);
    the getter reports the FFT window width W as its width, as the reference
    does (digHolo.cpp:4362-4380).  The batch-sum intensity has a stride of
    W H floats per polarisation, of which the first (W/2+1) H are the plane's."""
    b, p, w, hh = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    fp = L.digHoloGetFourierPlaneFull(h, C.byref(b), C.byref(p), C.byref(w), C.byref(hh))
    out = {}
    if fp and w.value > 0:
        nxr = w.value // 2 + 1
        n = b.value * p.value * hh.value * nxr
        out["plane"] = np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64).reshape(
            b.value, p.value, hh.value, nxr)
        out["width"] = w.value
    pcount, tcount, pcn = C.c_int(), C.c_int(), C.c_int()
    params = C.POINTER(C.c_float)()
    px, py = C.c_int(), C.c_int()
    xa, ya, ti = C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    rc = L.digHoloBatchGetSummary(h, 0, C.byref(pcount), C.byref(tcount), C.byref(pcn), C.byref(params),
                                  C.byref(px), C.byref(py), C.byref(xa), C.byref(ya), C.byref(ti))
    out["summary_rc"] = rc
    if rc == 0:
        stats = np.ctypeslib.as_array(params, shape=(pcount.value * pcn.value * tcount.value,)).copy()
        out["summary"] = stats.reshape(pcount.value, pcn.value, tcount.value)
        out["px"], out["py"] = px.value, py.value
        W = 2 * (px.value - 1)
        stride = W * py.value
        tot = np.ctypeslib.as_array(ti, shape=(pcn.value * stride,)).copy().reshape(pcn.value, stride)
        out["batchsum"] = tot[:, :px.value * py.value].reshape(pcn.value, py.value, px.value)
        out["kx"] = np.ctypeslib.as_array(xa, shape=(W,)).copy()
        out["ky"] = np.ctypeslib.as_array(ya, shape=(py.value,)).copy()
    return out
