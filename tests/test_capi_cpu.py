"""C ABI checks that need no GPU: exported symbols and host-side error paths."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO

from ho2d import capi, meshgen

HEADER = os.path.join(REPO, "include", "ho2d.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ho2d_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in capi.SIGNATURES, n


def _handle():
    lib = capi.load()
    h = ctypes.c_void_p()
    assert lib.ho2d_create(ctypes.byref(h)) == 0
    return lib, h


def test_null_and_order_errors(tmp_path):
    lib, h = _handle()
    try:
        assert lib.ho2d_setup(None) == 1
        assert lib.ho2d_setup(h) == 1  # before read_input
        assert b"read_input" in lib.ho2d_last_error(h)
        assert lib.ho2d_step(h, 1) == 1
        buf = np.zeros(4)
        assert lib.ho2d_get_vort(h, 4, capi.dptr(buf)) == 1
    finally:
        lib.ho2d_destroy(h)


def test_missing_input_file(tmp_path):
    lib, h = _handle()
    try:
        assert lib.ho2d_read_input(h, str(tmp_path / "nope.dat").encode()) == 2
    finally:
        lib.ho2d_destroy(h)


@pytest.mark.parametrize("field,value,code", [(1, "9", 4), (9, "3", 4), (10, "7", 4), (11, "3", 4), (12, "16", 4)])
def test_unsupported_settings(tmp_path, field, value, code):
    path = meshgen.make_case("cavity4", str(tmp_path), steps=1)
    lines = open(path).read().split("\n")
    # value lines: Knod at 3; huynh at 19; time integration 21; advection 23; problem type 25
    idx = {1: 3, 9: 19, 10: 21, 11: 23, 12: 25}[field]
    lines[idx] = value
    open(path, "w").write("\n".join(lines))
    lib, h = _handle()
    try:
        assert lib.ho2d_read_input(h, path.encode()) == code
    finally:
        lib.ho2d_destroy(h)


def _setup_code(path):
    lib, h = _handle()
    try:
        assert lib.ho2d_read_input(h, path.encode()) == 0
        return lib.ho2d_setup(h), lib.ho2d_last_error(h)
    finally:
        lib.ho2d_destroy(h)


def test_mesh_errors(tmp_path):
    path = meshgen.make_case("cavity4", str(tmp_path), steps=1)
    msh = os.path.join(str(tmp_path), "mesh.msh")
    good = open(msh).read()
    # unsupported quad type
    open(msh, "w").write(good.replace("2 1 3 16", "2 1 99 16"))
    code, msg = _setup_code(path)
    assert code == 3 and b"unsupported" in msg
    # missing section
    open(msh, "w").write(good.replace("$Elements", "$Elementz"))
    code, _ = _setup_code(path)
    assert code == 3
    # a boundary curve left out: its element sides have no boundary edge
    lines = good.split("\n")
    i = lines.index("1 1 1 4")
    open(msh, "w").write("\n".join(lines[:i] + lines[i + 5:]).replace("5 36 1 36", "5 32 1 36"))
    code, _ = _setup_code(path)
    assert code == 3


def test_valid_mesh_reaches_device_setup(tmp_path):
    """Host parsing and setup succeed; only the CUDA part may fail without a GPU."""
    path = meshgen.make_case("cyl4x8", str(tmp_path), steps=1)
    code, msg = _setup_code(path)
    assert code in (0, 5), msg


def test_precision_modes():
    lib, h = _handle()
    try:
        for mode in (capi.FP64, capi.MIXED, capi.MIXED_KRYLOV):
            assert lib.ho2d_set_precision(h, mode) == capi.HO2D_OK
        assert lib.ho2d_set_precision(h, 3) == 1  # HO2D_ERR_ARG
        assert b"HO2D_MIXED_KRYLOV" in lib.ho2d_last_error(h)
    finally:
        lib.ho2d_destroy(h)


def test_forces_need_setup():
    lib, h = _handle()
    try:
        fx, fy = ctypes.c_double(), ctypes.c_double()
        assert lib.ho2d_get_forces(h, ctypes.byref(fx), ctypes.byref(fy)) == 1
        assert b"set up" in lib.ho2d_last_error(h)
    finally:
        lib.ho2d_destroy(h)


def _cli():
    import shutil

    if shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
        pytest.skip("nvcc not available to link the CLI")
    from ho2d import build

    build.build(cli=True)
    return os.path.join(os.path.dirname(build.LIB), "ho2d_main")


def test_cli_arguments_and_input_errors(tmp_path):
    """The command-line drop-in for src/main.cpp: usage on an unknown option, the input
    reader's error code for a missing file and for an unsupported setting; none of these
    reach the device."""
    import subprocess

    exe = _cli()
    r = subprocess.run([exe, "--bogus"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 255 and "Usage" in r.stdout
    r = subprocess.run([exe, str(tmp_path / "nope.dat")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and r.stdout.startswith("error 2:"), r.stdout
    path = meshgen.make_case("cavity4", str(tmp_path), steps=1)
    lines = open(path).read().split("\n")
    lines[21] = "7"  # time integration type 7 does not exist
    open(path, "w").write("\n".join(lines))
    r = subprocess.run([exe, path, "--mixed"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 4 and "error 4:" in r.stdout, r.stdout
