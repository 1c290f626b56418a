"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares."""
import ctypes
import os
import re

from .conftest import ROOT

HEADER_DIR = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "hos_b200", "libhos_gpu.so")


def declared_functions():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "return", "sizeof"):
                names.add(name)
    return names


def test_library_built():
    assert os.path.exists(LIB), "run make -C hos_b200/csrc"


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    names = declared_functions()
    assert "hos_create" in names and "hos_step" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_without_gpu():
    import hos_b200

    lib = hos_b200.load()
    assert b"sm_100a" in lib.hos_version()
    assert lib.hos_last_error() is not None


def test_footprint_scales():
    from hos_b200 import HosField

    a = HosField.footprint_bytes(256, 256, order=3)
    b = HosField.footprint_bytes(512, 512, order=3)
    c = HosField.footprint_bytes(512, 512, order=3, precision="fp32")
    assert 3.5 * a < b < 4.5 * a
    assert c < b
