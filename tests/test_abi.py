"""The C-ABI library builds, loads and exports every entry point that
include/scg.h declares (no device work)."""
import ctypes
import os
import re
import subprocess

import scgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "scg.h")).read()
    return sorted(set(re.findall(r"^int (scg_\w+)\(", src, re.M)))


def test_header_and_binding_agree():
    assert declared() == sorted(scgpu.EXPORTS)


def test_library_exports_every_symbol():
    lib = scgpu.load()
    out = subprocess.run(["nm", "-D", "--defined-only", scgpu.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    syms = set(l.split()[-1] for l in out.splitlines() if l.strip())
    for name in declared():
        assert name in syms, name
        assert getattr(lib, name) is not None


def test_errors_are_reported_not_raised_in_c():
    lib = scgpu.load()
    buf = ctypes.create_string_buffer(256)
    assert lib.scg_index_destroy(None) == 0
    assert lib.scg_precompute(None) == -1
    assert lib.scg_last_error(buf, 256) == 0
    assert b"null" in buf.value
