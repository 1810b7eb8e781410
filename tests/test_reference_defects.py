"""Defects of the reference build that this build does not reproduce, shown
on the reference compiled from its sources (oracle/_ref).

* convert_int16tofloat32 with transpose (digHolo.cpp:1206-1229) is meant to
  transpose each frame (digHolo.h:265), but its lane permutation (0xDB where
  its own comment reads 0b11011000) scrambles every even output row: row 1 of
  a transposed 16 x 16 frame is column 1 of the input, row 0 is not column 0.
"""
import ctypes as C

import numpy as np
import pytest

import ref_lib


def _aligned(n, dtype, a=64):
    buf = np.zeros(n * np.dtype(dtype).itemsize + a, dtype=np.uint8)
    off = (-buf.ctypes.data) % a
    return buf[off:off + n * np.dtype(dtype).itemsize].view(dtype)


def test_reference_transposing_converter_scrambles_even_rows():
    if not ref_lib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    lib = C.CDLL(ref_lib.LIB_PATH)
    f = getattr(lib, "_Z22convert_int16tofloat32PtPfiiiih")
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ubyte]
    N = 16
    p = _aligned(N * N, np.uint16)
    p[:] = np.arange(N * N)
    out = _aligned(N * N, np.float32)
    f(p.ctypes.data, out.ctypes.data, 0, N, N, N, 1)
    rows = out.astype(int).reshape(N, N)
    src = p.astype(int).reshape(N, N)
    for i in range(1, N, 2):
        np.testing.assert_array_equal(rows[i], src[:, i])      # odd rows: the transpose
    assert not np.array_equal(rows[0], src[:, 0])              # even rows: scrambled
