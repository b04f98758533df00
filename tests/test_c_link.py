"""CPU test: a C program includes blasx_b200.h after a CBLAS_H-guarded
cblas.h, links -lblasx_b200 like a BLASX user, and gets the reference's
error behaviour (no GPU needed)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_program_links_and_reports(blx, tmp_path):
    exe = tmp_path / "link_check"
    libdir = os.path.dirname(blx.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c", "link_check.c"), "-L", libdir, "-lblasx_b200",
                        f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES="")).stdout
    assert " ** On entry to DGEMM  parameter number  8 had an illegal value\n" in out
    assert " ** On entry to DGEMM  parameter number  1 had an illegal value\n" in out
    assert " ** On entry to DSYRK  parameter number 10 had an illegal value\n" in out
    assert " ** On entry to DSYMM  parameter number  9 had an illegal value\n" in out
    assert " ** On entry to  ZHEMM parameter number  1 had an illegal value\n" in out
    assert " ** On entry to DTRMM  parameter number  4 had an illegal value\n" in out
    assert " ** On entry to DTRSM  parameter number 11 had an illegal value\n" in out
    assert " ** On entry to DTRSM  parameter number  1 had an illegal value\n" in out
    assert "status=1" in out and "status=0 C0=1" in out
    assert "plan rc=0 loads=200 min_ratio=1.000" in out
