"""C-ABI library checks that need no GPU: it builds, loads and exports every
entry point include/magic_b200.h declares; the ctypes prototypes match."""

import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "magic_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mt_[A-Za-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def libpath():
    from magic_b200.csrc import build

    return build.build()


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mt_[A-Za-z0-9_]+)", out))
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [s for s in declared if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    # nothing but the C ABI is visible
    assert all(s.startswith("mt_") for s in exported)


def test_ctypes_prototypes_cover_header(libpath):
    from magic_b200 import _lib

    L = _lib.lib()
    assert set(_lib.EXPORTED) == set(_declared())
    for name in _lib.EXPORTED:
        assert getattr(L, name) is not None


def test_struct_layouts_match_header(libpath, tmp_path):
    """Compile a tiny C program against the header and compare sizeof/offsetof."""
    from magic_b200 import _lib

    structs = {"mt_grid_desc": _lib.GridDesc, "mt_plan_info": _lib.PlanInfo,
               "mt_anel_params": _lib.AnelParams, "mt_courant_params": _lib.CourantParams,
               "mt_bouss_in": _lib.BoussIn, "mt_bouss_out": _lib.BoussOut,
               "mt_bouss_params": _lib.BoussParams, "mt_anel_in": _lib.AnelIn,
               "mt_anel_out": _lib.AnelOut, "mt_anel_stage_params": _lib.AnelStageParams,
               "mt_td_in": _lib.TdIn, "mt_td_out": _lib.TdOut, "mt_td_params": _lib.TdParams,
               "mt_field_update": _lib.FieldUpdate, "mt_am_correction": _lib.AmCorrection,
               "mt_poloidal_update": _lib.PoloidalUpdate, "mt_level_copy": _lib.LevelCopy}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(c)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_plan_create_rejects_bad_arguments(libpath):
    from magic_b200 import _lib

    L = _lib.lib()
    h = ctypes.c_void_p()
    desc = _lib.GridDesc(0, 1, 0, 0, 0)
    assert L.mt_plan_create(ctypes.byref(desc), ctypes.byref(h)) == 1  # MT_ERR_ARG
    assert b"l_max" in L.mt_last_error()
    desc = _lib.GridDesc(16, 1, 0, 0, 7)
    assert L.mt_plan_create(ctypes.byref(desc), ctypes.byref(h)) == 3  # unsupported precision
    assert L.mt_plan_destroy(None) == 0
    assert L.mt_transform_workspace(None, 4, 1) == 0


def test_radial_op_rejects_bad_arguments(libpath):
    """Argument checks of the radial-operator constructor run before any device call."""
    from magic_b200 import _lib

    L = _lib.lib()
    h = ctypes.c_void_p()
    D = (ctypes.c_double * 4)(1.0, 0.0, 0.0, 1.0)
    assert L.mt_radial_op_create(1, D, ctypes.byref(h)) == 1
    assert L.mt_radial_op_create(2, None, ctypes.byref(h)) == 1
    bad = (ctypes.c_double * 4)(1.0, float("nan"), 0.0, 1.0)
    assert L.mt_radial_op_create(2, bad, ctypes.byref(h)) == 1
    assert b"finite" in L.mt_last_error()
    assert L.mt_radial_op_create_dct1(1, ctypes.byref(h)) == 1
    assert L.mt_radial_op_destroy(None) == 0
    assert L.mt_radial_op_bandwidth(None) == 0
    M = (ctypes.c_double * 8)(*([1.0] * 8))
    assert L.mt_lop_create(0, 2, M, ctypes.byref(h)) == 1
    bad = (ctypes.c_double * 8)(*([1.0] * 7 + [float("inf")]))
    assert L.mt_lop_create(2, 2, bad, ctypes.byref(h)) == 1
    assert L.mt_lop_destroy(None) == 0


def test_no_cpu_fallback_without_gpu(libpath):
    """Without a GPU the product path refuses loudly instead of computing on the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from magic_b200 import Plan

    with pytest.raises(RuntimeError):
        Plan(16)


def test_device_status_codes_decode():
    from magic_b200 import MagicError, _lib

    assert _lib.describe_status(0) == "ok"
    assert "code 4" in _lib.describe_status(4)
    assert "synthesis" in _lib.describe_status(4)
    assert "code 12345" in _lib.describe_status(12345)
    _lib.raise_device_status(0)
    with pytest.raises(MagicError, match="invalid"):
        _lib.raise_device_status(14, "nl_bouss")


def test_device_status_rejects_null_arguments(libpath):
    from magic_b200 import _lib

    L = _lib.lib()
    code = ctypes.c_int(0)
    assert L.mt_device_status(None, ctypes.byref(code), None) != 0
    assert L.mt_noalloc_status(None, None) != 0
