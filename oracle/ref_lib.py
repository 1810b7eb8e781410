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



# The reference exposes the same C ABI, so the product's numpy helpers drive it too.
from digholo_b200.api import configure, run_batch, set_batch, read_outputs, ptr  # noqa: E402,F401
