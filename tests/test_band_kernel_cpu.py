"""The direct solver's banded block-Cholesky kernel (k_band_solve in
colb_b200/csrc/dense.cu), run from its own source on the CPU.

The kernel text is cut out of dense.cu, compiled with g++ against a host
emulation of the CUDA thread model (tests/simt/simt.h: one std::thread per
CUDA thread, the two CTAs of a cluster at the same time, barriers for
__syncthreads / __syncwarp / the named and cluster barriers, an exchange
array for __shfl_sync) and run on random SPD block-band matrices of 2 to 46
bodies and body bandwidths 1 to 8 (the window wraps once a component is
wider than its band; components of at least 2 wb + 12 bodies are split
between the two CTAs of their cluster and meet at a separator).  Every
solution must match a dense Cholesky solve to 1e-12 relative.  This checks
the kernel's indexing, phases and barriers without a GPU; the GPU tests
check the compiled kernel inside the solver."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _kernel_source():
    src = open(os.path.join(ROOT, "colb_b200", "csrc", "dense.cu")).read()
    k = src[src.index("constexpr int BAND_MAX = 8;"):src.index("struct DenseState {")]
    k = k.replace("extern __shared__ __align__(16) unsigned char smem_raw[];", "unsigned char* smem_raw = g_dyn_smem;")
    # the gather kernel reads the block CSR of the engine: not needed here
    return k[:k.index("template <class TV>")] + k[k.index("// Warp-wide Cholesky factorization and inversion"):]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_band_kernel_source_solves_block_band_systems(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "band_kernel.inc"), "w").write(_kernel_source())
    for f in ("simt.h", "band_test.cpp"):
        shutil.copy(os.path.join(HERE, "simt", f), d)
    exe = os.path.join(d, "band_test")
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-pthread", os.path.join(d, "band_test.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "status 0" in out.stdout and "split 5" in out.stdout
