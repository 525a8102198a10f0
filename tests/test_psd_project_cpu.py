"""The warp-level PSD projection of the contact Hessians
(colb_b200/csrc/warp_eig.cuh), run from its own source on the CPU.

The header is compiled with g++ against the host emulation of the CUDA
thread model (tests/simt/simt.h: one std::thread per CUDA thread, warp
shuffles and votes through a per-warp array) and the register-resident
projection (one lane per row, warp_psd_project_rows) is compared with the
shared-memory one (team_psd_project, which the GPU tests check against the
oracle) on indefinite, rank-deficient, positive-definite and zero matrices
of sizes 6, 9 and 12: equal to 1e-12 of the matrix scale, symmetric, and
positive semidefinite."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _header_source():
    src = open(os.path.join(ROOT, "colb_b200", "csrc", "warp_eig.cuh")).read()
    return src.replace('#include "common.cuh"', "").replace("#pragma once", "")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_register_projection_matches_shared_memory_projection(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "warp_eig.inc"), "w").write(_header_source())
    for f in ("simt.h", "eig_test.cpp"):
        shutil.copy(os.path.join(HERE, "simt", f), d)
    exe = os.path.join(d, "eig_test")
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-pthread", os.path.join(d, "eig_test.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ok" in out.stdout
