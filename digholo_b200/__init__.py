"""digholo_b200: the digHolo batch path (FFT -> window -> IFFT -> tilt ->
HG overlap, plus AutoAlign metrics) as sm_100a CUDA kernels behind the
digHolo C ABI.

The product is the shared library ``libdigholo_b200.so`` built in this
directory (see csrc/Makefile); this package only binds it with ctypes.
There is no CPU fallback: :func:`load` raises if the library is missing, and
the library's processing entry points fail when no CUDA device is present.
"""
import ctypes as _C
import os as _os

from . import abi

HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(HERE, "libdigholo_b200.so")

_LIB = None
_BOUND = None


def load():
    """Load libdigholo_b200.so once and return its bound entry points."""
    global _LIB, _BOUND
    if _BOUND is None:
        if not _os.path.exists(LIB_PATH):
            raise ImportError("libdigholo_b200.so is not built: run `make -C digholo_b200/csrc` "
                              "(or __graft_entry__.build())")
        _LIB = _C.CDLL(LIB_PATH)
        _BOUND = abi.bind(_LIB)
        _bind_extensions(_LIB, _BOUND)
    return _BOUND


def _bind_extensions(lib, out):
    P = _C.POINTER
    ext = {
        "digHoloB200ProcessBatchDevice": (_C.c_int, [_C.c_int]),
        "digHoloB200GetCoefsDevice": (P(_C.c_float), [_C.c_int, P(_C.c_int), P(_C.c_int), P(_C.c_int)]),
        "digHoloB200Synchronize": (_C.c_int, [_C.c_int]),
        "digHoloB200SetKeepField32": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200GetFields32": (P(_C.c_float), [_C.c_int, P(_C.c_int), P(_C.c_int), P(_C.c_int), P(_C.c_int)]),
        "digHoloB200GetLastError": (_C.c_char_p, [_C.c_int]),
        "digHoloB200SetStream": (_C.c_int, [_C.c_int, _C.c_void_p]),
        "digHoloB200SetTiming": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200SetGraphs": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200GetGraphCount": (_C.c_int, [_C.c_int]),
        "digHoloB200GetStageTimes": (_C.c_int, [_C.c_int, P(_C.c_float)]),
        "digHoloB200GetGeometry": (_C.c_int, [_C.c_int, P(_C.c_int)]),
        "digHoloB200SetForwardKernel": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200GetAutoAlignEvaluations": (_C.c_int, [_C.c_int]),
        "digHoloB200GetForwardKernel": (_C.c_int, [_C.c_int]),
        "digHoloB200SetInverseKernel": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200GetInverseKernel": (_C.c_int, [_C.c_int]),
        "digHoloB200SetOverlapKernel": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200GetOverlapKernel": (_C.c_int, [_C.c_int]),
        "digHoloB200AutoAlignGradient": (_C.c_int, [_C.c_int, P(_C.c_float), P(_C.c_float)]),
        "digHoloB200AutoAlignAdjoint": (_C.c_float, [_C.c_int]),
        "digHoloB200AutoAlignGradientMetric": (_C.c_int, [_C.c_int, _C.c_int, P(_C.c_float), P(_C.c_float)]),
        "digHoloB200FreezeWindow": (_C.c_int, [_C.c_int, _C.c_int]),
        "digHoloB200GetKernelPlan": (_C.c_int, [_C.c_int, P(_C.c_int), P(_C.c_int), P(_C.c_float)]),
        "digHoloB200GetKernelPlanRuns": (_C.c_int, []),
        "digHoloB200EigenHermitian": (_C.c_int, [_C.c_int, P(_C.c_double), P(_C.c_double), P(_C.c_double)]),
        "digHoloB200FrameSimulatorDevice": (_C.c_int, [_C.c_int, _C.c_int, _C.c_int, _C.c_float, _C.c_int] +
                                            [P(_C.c_float)] * 6 + [_C.c_int] + [P(_C.c_float)] * 4 +
                                            [_C.c_int, _C.c_int, P(_C.c_float), _C.c_int, _C.c_void_p, _C.c_void_p]),
        "digHoloB200ProcessBatchNoAlloc": (_C.c_int, [_C.c_int, _C.c_void_p, _C.c_int, _C.c_int, _C.c_void_p,
                                                     _C.c_void_p, _C.c_void_p, _C.c_void_p]),
    }
    for name, (ret, args) in ext.items():
        fn = getattr(lib, name, None)
        if fn is None:
            out.missing.append(name)
            continue
        fn.restype = ret
        fn.argtypes = args
        setattr(out, name, fn)
