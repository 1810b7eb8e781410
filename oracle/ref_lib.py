"""ctypes binding of the compiled digHolo reference (oracle/_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's reference / cpu_baseline leg, never by the product.

oracle/Makefile compiles the unmodified reference sources (digHolo.cpp,
digHolo.h) with this project's shims into _ref/libdigholo_ref.so and writes
_ref/symbols.txt (mangled name <TAB> demangled signature).  The reference's
Linux exports are C++-mangled (EXT_C is empty there, digHolo.h:148-156), so
entry points are found through that map and typed with the shared
prototype table in digholo_b200/abi.py.
"""
import ctypes as C
import os

from digholo_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libdigholo_ref.so")
SYMBOLS_PATH = os.path.join(HERE, "_ref", "symbols.txt")


def available():
    return os.path.exists(LIB_PATH) and os.path.exists(SYMBOLS_PATH)


def _symbol_map():
    table = {}
    with open(SYMBOLS_PATH) as f:
        for line in f:
            parts = line.rstrip("\n").split("\t")
            if len(parts) != 2:
                continue
            mangled, demangled = parts
            name = demangled.split("(")[0].strip()
            if "::" in name or " " in name:
                continue
            table.setdefault(name, mangled)
    return table


_LIB = None


def load():
    """Load the reference library once and return its bound entry points."""
    global _LIB
    if _LIB is None:
        if not available():
            raise FileNotFoundError("reference build missing: run `make -C oracle` where the reference sources exist")
        lib = C.CDLL(LIB_PATH)
        table = _symbol_map()
        _LIB = abi.bind(lib, resolver=table.get)
    return _LIB


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def configure(L, h, cfg):
    """Apply an oracle Config to a digHolo handle through the C ABI setters."""
    L.digHoloConfigSetFrameDimensions(h, cfg.frame_width, cfg.frame_height)
    L.digHoloConfigSetFramePixelSize(h, float(cfg.pixel_size))
    L.digHoloConfigSetWavelengthCentre(h, float(cfg.wavelength))
    L.digHoloConfigSetPolCount(h, cfg.pol_count)
    L.digHoloConfigSetfftWindowSize(h, int(cfg.fft_window[0]), int(cfg.fft_window[1]))
    L.digHoloConfigSetFourierWindowRadius(h, float(cfg.window_radius_deg))
    L.digHoloConfigSetIFFTResolutionMode(h, cfg.resolution_mode)
    L.digHoloConfigSetBasisGroupCount(h, cfg.max_mg)
    L.digHoloConfigSetFillFactorCorrectionEnabled(h, cfg.fill_factor)
    L.digHoloConfigSetPolLockTilt(h, cfg.pol_lock_tilt)
    L.digHoloConfigSetPolLockDefocus(h, cfg.pol_lock_defocus)
    L.digHoloConfigSetPolLockBasisWaist(h, cfg.pol_lock_waist)
    for p in range(cfg.pol_count):
        L.digHoloConfigSetBasisWaist(h, p, float(cfg.waist[p]))
        L.digHoloConfigSetBeamCentre(h, 0, p, float(cfg.beam_centre[p][0]))
        L.digHoloConfigSetBeamCentre(h, 1, p, float(cfg.beam_centre[p][1]))
        L.digHoloConfigSetTilt(h, 0, p, float(cfg.tilt_deg[p][0]))
        L.digHoloConfigSetTilt(h, 1, p, float(cfg.tilt_deg[p][1]))
        L.digHoloConfigSetDefocus(h, p, float(cfg.defocus[p]))


def run_batch(L, h, frames):
    """SetBatch(Uint16) + ProcessBatch; returns the outputs as numpy copies.

    Keys: coefs (B, P, M) complex64 (or None), field (B, P, ny, nx) complex64,
    R / I int16 (B, P, ny, nx), scale (P, B) float32, x, y axes.
    """
    import numpy as np
    frames = np.ascontiguousarray(frames)
    B = frames.shape[0]
    if frames.dtype == np.uint16:
        L.digHoloSetBatchUint16(h, B, ptr(frames, C.c_ushort), 0)
    else:
        frames = frames.astype(np.float32, copy=False)
        L.digHoloSetBatch(h, B, ptr(frames, C.c_float))
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    cp = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    out = {}
    if cp and m.value > 0:
        arr = np.ctypeslib.as_array(cp, shape=(b.value * pc.value * m.value * 2,)).copy()
        out["coefs"] = arr.view(np.complex64).reshape(b.value, pc.value, m.value)
    else:
        out["coefs"] = None
    fr = C.POINTER(C.c_short)()
    fi = C.POINTER(C.c_short)()
    fs = C.POINTER(C.c_float)()
    x = C.POINTER(C.c_float)()
    y = C.POINTER(C.c_float)()
    w, hh = C.c_int(), C.c_int()
    L.digHoloGetFields16(h, C.byref(b), C.byref(pc), C.byref(fr), C.byref(fi), C.byref(fs),
                         C.byref(x), C.byref(y), C.byref(w), C.byref(hh))
    n = b.value * pc.value * w.value * hh.value
    shape = (b.value, pc.value, hh.value, w.value)
    out["R"] = np.ctypeslib.as_array(fr, shape=(n,)).copy().reshape(shape)
    out["I"] = np.ctypeslib.as_array(fi, shape=(n,)).copy().reshape(shape)
    out["x"] = np.ctypeslib.as_array(x, shape=(w.value,)).copy()
    out["y"] = np.ctypeslib.as_array(y, shape=(hh.value,)).copy()
    fp = L.digHoloGetFields(h, C.byref(b), C.byref(pc), C.byref(x), C.byref(y), C.byref(w), C.byref(hh))
    out["field"] = np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64).reshape(shape)
    # DIGHOLO_ANALYSIS[IFFT][MAXABS][pol][batch]: through BatchGetSummary(plane 1)
    pcount, tcount, pcn = C.c_int(), C.c_int(), C.c_int()
    params = C.POINTER(C.c_float)()
    px, py = C.c_int(), C.c_int()
    xa, ya, ti = C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    L.digHoloBatchGetSummary(h, 1, C.byref(pcount), C.byref(tcount), C.byref(pcn), C.byref(params),
                             C.byref(px), C.byref(py), C.byref(xa), C.byref(ya), C.byref(ti))
    stats = np.ctypeslib.as_array(params, shape=(pcount.value * pcn.value * tcount.value,)).copy()
    out["summary"] = stats.reshape(pcount.value, pcn.value, tcount.value)
    out["scale"] = out["summary"][3, :, :B]
    return out
