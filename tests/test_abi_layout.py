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
