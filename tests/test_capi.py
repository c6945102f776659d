"""CPU tests of the boundary: libklft_b200.so loads, exports every entry point
declared in include/klft_b200.h, and fails loudly (no CPU fallback) when no
CUDA device is present."""
import ctypes
import os
import re

import pytest

from tests.conftest import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(klft_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from klft_b200._lib import LIB_PATH, SIGNATURES
    lib = ctypes.CDLL(LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers every declared entry point
    assert not [n for n in names if n not in SIGNATURES], [n for n in names if n not in SIGNATURES]


def test_version_and_errors_without_compute():
    from klft_b200._lib import lib
    assert lib().klft_version() >= 100
    # invalid arguments are rejected before any device work
    h = ctypes.c_void_p()
    L = (ctypes.c_int * 4)(4, 4, 4, 4)
    assert lib().klft_lattice_create(4, 4, L, 0, 0, 0, ctypes.byref(h)) == 1  # Nc = 4 unsupported
    assert b"Nc" in lib().klft_last_error()
    L = (ctypes.c_int * 4)(4, 5, 4, 4)
    assert lib().klft_lattice_create(3, 4, L, 0, 0, 0, ctypes.byref(h)) == 1  # odd extent
    assert lib().klft_plaquette(None, None) == 1


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_cpu_fallback():
    import klft_b200
    with pytest.raises(klft_b200.KlftError) as e:
        klft_b200.GaugeField([4, 4, 4, 4], 3)
    assert "KLFT_ECUDA" in str(e.value)
