"""The PETSc MATSHELL adapter (parallel-computing_b200/adapters/petsc_matshell.cpp).

The adapter is the source file a maintainer adds to the reference's PETSc
drivers so that their MATSHELL MatMult (matrix_free/iteration_number_fempc_mf.cpp:
46-60, and its ghosted multi-rank layout, :62-72) calls this library. PETSc is
not available here, so the test compiles the adapter against a stand-in of the
few PETSc and CUDA runtime declarations it uses (tests/petsc_mock/) and fake
library entry points, and checks what it does: the device or host arrays it
hands to iga_apply / iga_apply_host, a failing status turned into
PETSC_ERR_LIB with the library's message, and the ghosted MatMult's order
(forward ghost update, iga_part_apply on the local forms, reverse add of the
ghost rows), plus the ghosted vectors' layout.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_matshell_adapter_against_petsc_standin(tmp_path):
    exe = tmp_path / "adapter_driver"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-Wno-unused-parameter",
           "-I", os.path.join(ROOT, "tests", "petsc_mock"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "petsc_mock", "adapter_driver.cpp"),
           os.path.join(ROOT, "parallel-computing_b200", "adapters", "petsc_matshell.cpp"), "-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
    assert run.stdout.strip().endswith("ok")
