"""libjuicer_b200.so loads without a GPU and exports every function that
include/*.h declares; the Python bindings declare exactly that set (no compute call
is made here)."""
import ctypes as C
import os
import re

import film_juicer_b200 as pkg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][A-Za-z0-9_]*\s*\**\s+(fjb?_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(pkg.LIB_PATH)
    declared = _declared()
    assert {"fj_cuda_create", "fj_cuda_render", "fj_cuda_destroy", "fjb_render_pixels"} <= declared
    for name in declared:
        assert hasattr(lib, name), name


def test_python_bindings_cover_the_headers():
    assert _declared() == set(pkg.exported_names())


def test_load_library_declares_signatures():
    lib = pkg.load_library()
    assert lib.fj_cuda_render.restype is not None
