"""The C-ABI library builds, loads and exports every symbol its header declares.

No compute call is made here (no GPU needed)."""
import ctypes
import os
import re

from hydra_b200 import build as hb_build
from hydra_b200 import casl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"^[a-z_ ]+\**\s*\**(casl_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_header_symbols():
    path = hb_build.build()
    lib = ctypes.CDLL(path)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) <= set(casl.SIGNATURES)


def test_error_strings():
    lib = casl.load_library(hb_build.build())
    assert lib.casl_error_string(0) == b"ok"
    assert b"capacity" in lib.casl_error_string(2)


def test_create_rejects_bad_parameters_without_gpu_work():
    lib = casl.load_library(hb_build.build())
    p = casl.CaslParams(100, 100, 10, 6.28, 6.28, 0, 0, 0, 0, 2, 3, 0, 0, 0, 0, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    assert lib.casl_create(ctypes.byref(p), 0, ctypes.byref(h)) == casl.CASL_EINVAL
