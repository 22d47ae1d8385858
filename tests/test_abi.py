"""The C ABI: the library loads without a GPU, exports every symbol include/retainwall.h
declares, and its ctypes mirror matches the header's struct layouts.  No compute call."""
import ctypes as ct
import os
import re

import pytest

from retainwall_code_b200 import _abi, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "retainwall.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rw_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_abi():
    fns = header_functions()
    assert "rw_create" in fns and "rw_step" in fns and len(fns) >= 20


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [f for f in header_functions() if not hasattr(L, f)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == sorted(header_functions())


def test_struct_sizes_match_header():
    # offsets computed by the C compiler for the header structs
    import subprocess, tempfile

    code = r'''
#include <stdio.h>
#include <stddef.h>
#include "retainwall.h"
int main(){printf("%zu %zu %zu %zu %zu %zu\n", sizeof(rw_motion), sizeof(rw_case_params), sizeof(rw_case),
 sizeof(rw_info), offsetof(rw_case_params, model_par), offsetof(rw_case_params, motion));return 0;}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(code)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    want = [ct.sizeof(_abi.Motion), ct.sizeof(_abi.CaseParams), ct.sizeof(_abi.Case), ct.sizeof(_abi.Info),
            _abi.CaseParams.model_par.offset, _abi.CaseParams.motion.offset]
    assert got == want


def test_status_strings():
    L = _lib.lib()
    assert L.rw_status_string(0) == b"RW_OK"
    assert L.rw_status_string(7) == b"RW_EDEVICE"
    assert L.rw_status_string(99) == b"RW_UNKNOWN"


def test_create_missing_project_reports_enoent(tmp_path):
    L = _lib.lib()
    h = ct.c_void_p()
    st = L.rw_create(str(tmp_path / "nope").encode(), 0, 4, ct.byref(h))
    assert st == _abi.RW_ENOENT
    assert b"Cannot load" in L.rw_last_error(None)
    assert not h.value


def test_create_missing_tag_reports_eformat(tmp_path):
    from retainwall_code_b200 import cases as C

    case = C.column_collapse(nx=4, ny=4, nz=4, runout=0.5)
    proj = str(tmp_path / "p")
    C.write_case(case, proj)
    txt = open(proj + ".xml").read().replace('  <cfl-number type="scalar">0.100000001</cfl-number>\n', "")
    open(proj + ".xml", "w").write(txt)
    L = _lib.lib()
    h = ct.c_void_p()
    st = L.rw_create(proj.encode(), 0, 4, ct.byref(h))
    assert st == _abi.RW_EFORMAT
    assert b"cfl-number does not exist" in L.rw_last_error(None)


def test_bad_precision_and_null_args():
    L = _lib.lib()
    h = ct.c_void_p()
    assert L.rw_create(b"x", 0, 3, ct.byref(h)) in (_abi.RW_EINVAL, _abi.RW_ENOENT)
    assert L.rw_step(None, 1) == _abi.RW_EINVAL
    assert L.rw_destroy(None) == _abi.RW_EINVAL
