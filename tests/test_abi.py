"""The C-ABI library loads and exports every entry point include/
wakis_b200.h declares; host-side argument checks reject bad descriptors
(no kernel is launched by these calls)."""

import ctypes
import os
import re

import pytest

from wakis_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "wakis_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wk_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_native.LIB_PATH):
        from wakis_b200 import build
        build.build(verbose=False)
    return _native.lib()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert names, "no declarations parsed"
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_native.EXPORTED)


def test_version(lib):
    assert lib.wk_version() == 1


def test_null_descriptor_rejected(lib):
    rc = lib.wk_fit_step(None, 1, 0, None)
    assert rc == 1
    assert b"descriptor" in lib.wk_last_error()


def test_bad_shape_rejected(lib):
    d = _native.FitDesc()
    d.Nx, d.Ny, d.Nz = 1, 4, 4
    rc = lib.wk_fit_step(ctypes.byref(d), 1, 0, None)
    assert rc == 2
    with pytest.raises(ValueError):
        _native.check(rc, "wk_fit_step")


def test_wake_args_rejected(lib):
    assert lib.wk_wake_potential(None, 0, 1, 1, None, 1, 0, None, None, 0, 0, None, 0, None, 0,
                                 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0, None, None) == 1
    assert lib.wk_dft_bins(None, 1, 1, 1, 1, None, None) == 1


@pytest.mark.parametrize("cname,ctype", [("wk_fit_desc", _native.FitDesc),
                                          ("wk_batch_plan", _native.BatchPlan)])
def test_descriptor_layout_matches_header(tmp_path, cname, ctype):
    """ctypes struct offsets equal the C struct's (gcc offsetof)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    fields = [f[0] for f in ctype._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "wakis_b200.h"',
           'int main(void){', f'printf("size %zu\\n", sizeof({cname}));']
    src += [f'printf("{f} %zu\\n", offsetof({cname}, {f}));' for f in fields]
    src += ["return 0;}"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(c)],
                   check=True)
    out = dict(line.split() for line in
               subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    assert int(out["size"]) == ctypes.sizeof(ctype)
    for f in fields:
        assert int(out[f]) == getattr(ctype, f).offset, f


def test_batch_args_rejected(lib):
    """The batched entry points check their arguments on the host."""
    assert lib.wk_batch_workspace_bytes(None, 1) == -1
    assert b"descs" in lib.wk_last_error()
    d = (_native.FitDesc * 1)()
    assert lib.wk_batch_workspace_bytes(d, 0) == -1
    d[0].Nx, d[0].Ny, d[0].Nz = 1, 4, 4
    assert lib.wk_batch_workspace_bytes(d, 1) == -1
    plan = _native.BatchPlan()
    assert lib.wk_batch_prepare(d, 1, 0, None, 0, ctypes.byref(plan), None) == 1
    assert lib.wk_batch_run(None, 1, 0, None, 0, None) == 1
    # a plan that wk_batch_prepare did not fill
    plan.workspace = 128
    plan.variant = -1
    assert lib.wk_batch_run(ctypes.byref(plan), 1, 0, None, 0, None) == 6
