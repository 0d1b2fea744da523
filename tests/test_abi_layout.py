"""The ctypes records (what a Python/Rust/other FFI host binds) match the C headers'
layout exactly: sizeof of every record and offsetof of every field, as compiled by
the system C compiler. Mirrors the reference's own layout assertions
(rust/film-juicer-plugin/src/cuda/abi_tests.rs:489+)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from film_juicer_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_program():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "juicer_b200.h"', 'int main(void) {']
    for rec in abi.ALL_RECORDS:
        name = rec.__name__
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in rec._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    return "\n".join(lines)


def test_record_layouts_match_c(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(_c_program())
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for rec in abi.ALL_RECORDS:
        assert int(got[rec.__name__]) == C.sizeof(rec), rec.__name__
        for fname, _ in rec._fields_:
            assert int(got[f"{rec.__name__}.{fname}"]) == getattr(rec, fname).offset, f"{rec.__name__}.{fname}"


def test_prepared_host_data_is_large_and_aligned():
    assert C.sizeof(abi.FjPreparedHostData) % 8 == 0
    assert C.alignment(abi.FjPreparedHostData) == 8


def test_repository_header_matches_reference_header_layout(tmp_path):
    """Drop-in check: the repository's include/juicer_cuda_api.h lays out every record
    that the reference's native/juicer_cuda_api.h declares (42 records) with the same
    sizeof and the same offsetof for every field. The reference's numbers come from
    tests/golden/abi_layout_reference.json (written by tests/golden/make_golden.py by
    compiling the reference header with the system C compiler), so this runs without
    the reference tree."""
    import json

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    with open(os.path.join(ROOT, "tests", "golden", "abi_layout_reference.json")) as fh:
        ref = json.load(fh)
    by_name = {r.__name__: r for r in abi.ALL_RECORDS}
    assert len(ref["records"]) == 42
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "juicer_cuda_api.h"', 'int main(void) {']
    for name in ref["records"]:
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in by_name[name]._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "ref_layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "ref_layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {k: int(v) for k, v in (line.rsplit(" ", 1) for line in out if line)}
    assert got == ref["layout"]
    # every field the reference lays out is one the ctypes mirror binds, at the same offset
    for key, off in ref["layout"].items():
        if "." in key:
            rec, field = key.split(".", 1)
            assert getattr(by_name[rec], field).offset == off, key
        else:
            assert C.sizeof(by_name[key]) == off, key
