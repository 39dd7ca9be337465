"""The C ABI library: loads, exports every declared entry point, and fails
loudly (no CPU fallback) when no CUDA device is present."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from blood_network_b200 import amg


def _lib_path():
    if not os.path.exists(amg.LIB_PATH):
        from blood_network_b200.build import build
        build()
    return amg.LIB_PATH


def test_exports_every_declared_symbol():
    path = _lib_path()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = set(amg.exported_symbols())
    missing = declared - exported
    assert not missing, f"declared in include/amg_b200.h but not exported: {sorted(missing)}"
    # the reference's drop-in names are all present
    for name in ("amg_solver_create", "amg_solver_update", "amg_solver_set_matrix",
                 "amg_solver_set_smoother", "amg_solver_solve", "amg_solver_size",
                 "amg_solver_num_levels", "amg_solver_free", "rs_strength", "pmis_coarsening",
                 "hmis_coarsening", "rs_coarsening", "rs_standard_interpolation", "dcsr_rap",
                 "abyvg", "abyvam", "abyvcs", "vbya", "ichol_compute", "ichol_solve"):
        assert name in exported


def test_only_c_abi_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib_path()], capture_output=True,
                         text=True, check=True).stdout
    names = [line.split()[-1] for line in out.splitlines() if line.strip()]
    cxx = [n for n in names if n.startswith("_Z")]
    assert not cxx, f"C++ symbols leak through the ABI: {cxx[:5]}"


def test_default_options_and_null_handles():
    lib = amg.load_library()
    o = amg.default_options()
    assert o.threshold == 0.25 and o.min_size == 500 and o.coarsening == amg.COARSEN_PMIS
    assert o.smoother == amg.SMOOTHER_CF_GS and o.precision == amg.PREC_FP64
    lib.amg_solver_free(None)            # accepts NULL, like the reference
    assert lib.amg_solver_size(None) == 0
    assert lib.amg_solver_num_levels(None) == 0


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = amg.load_library()
    ia = np.array([0, 1], np.int32)
    ja = np.array([0], np.int32)
    v = np.array([1.0])
    h = lib.amg_solver_create(1, 1, amg._p(ia), amg._p(ja), amg._p(v), 0.25, 10, 20, 1)
    assert not h
    assert lib.amg_solver_last_status() == -8   # AMG_ERR_NO_DEVICE
    assert b"device" in lib.amg_solver_last_error()


def test_reference_style_c_caller_builds_and_links(tmp_path):
    """A C program written against the reference wrapper's API compiles
    against include/amg_b200.h and links with the library (no GPU needed to
    build; tests/c/drop_in_example.c)."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "blood_network_b200", "lib")
    exe = str(tmp_path / "drop_in_example")
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror",
                    os.path.join(root, "tests", "c", "drop_in_example.c"),
                    "-I" + os.path.join(root, "include"), "-L" + lib, "-lamg_b200",
                    "-Wl,-rpath," + lib, "-lm", "-o", exe], check=True, capture_output=True)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_reference_style_c_caller_runs(tmp_path):
    """The same C program runs on the GPU and reaches its residual."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "blood_network_b200", "lib")
    exe = str(tmp_path / "drop_in_example")
    subprocess.run(["gcc", "-std=c99", "-O2", os.path.join(root, "tests", "c",
                                                           "drop_in_example.c"),
                    "-I" + os.path.join(root, "include"), "-L" + lib, "-lamg_b200",
                    "-Wl,-rpath," + lib, "-lm", "-o", exe], check=True, capture_output=True)
    out = subprocess.run([exe, "20000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "relres=" in out.stdout
