"""The C ABI without a GPU: the library builds, loads, exports every symbol
include/abd_b200.h declares, and its structs have the header's layout."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from colb_b200 import _abi
from colb_b200.engine import EXPORTS, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s+(abd_[a-z0-9_]+)\s*\(", src, re.M)
    return sorted(set(names))


def test_header_and_binding_agree():
    assert set(header_functions()) == set(EXPORTS)


def test_library_exports_every_symbol(built_library):
    L = load_library(built_library)
    for name in header_functions():
        assert hasattr(L, name), name
    assert L.abd_abi_version() == 2


def test_default_params_are_reference_constants(built_library):
    from colb_b200.engine import default_params
    from colb_b200.params import REFERENCE
    p = default_params()
    d = _abi.params_to_dict(p)
    for k in ("dt", "kappa", "k_ortho", "dhat", "cand_dist", "barrier", "newton_tol", "newton_max_iter",
              "lin_tol", "ls_min_alpha", "pinned_diag", "ee_f32", "self_contact"):
        assert d[k] == pytest.approx(REFERENCE[k]), k
    assert list(d["gravity"]) == [0.0, -10.0, 0.0]


def test_create_without_device_fails_loudly(built_library):
    """On a machine with no GPU the library returns an error; it never
    computes anything on the host."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except Exception:
        pass
    from colb_b200 import scene as S, params as P
    from colb_b200.engine import Engine, AbdError
    with pytest.raises(AbdError) as ei:
        Engine(P.reference_params(), S.config1_cubes())
    assert ei.value.code in (_abi.ABD_ERR_NO_DEVICE, _abi.ABD_ERR_CUDA)


def test_struct_layout_matches_header():
    code = r'''
#include <stdio.h>
#include <stddef.h>
#include "abd_b200.h"
int main(void) {
  printf("%zu %zu %zu\n", sizeof(AbdParams), sizeof(AbdSceneDesc), sizeof(AbdStepStats));
  printf("%zu %zu %zu %zu\n", offsetof(AbdParams, lin_tol), offsetof(AbdParams, precision),
         offsetof(AbdParams, pinned_diag), offsetof(AbdParams, warm_start));
  printf("%zu %zu\n", offsetof(AbdSceneDesc, planes), offsetof(AbdStepStats, gpu_ms));
  printf("%zu %zu %zu %zu\n", offsetof(AbdParams, ccd_max_iter), offsetof(AbdParams, test_inject),
         offsetof(AbdStepStats, solver_capped), offsetof(AbdStepStats, host_syncs));
  return 0; }
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c"); exe = os.path.join(d, "t")
        open(src, "w").write(code)
        cc = "x86_64-linux-gnu-gcc-13" if subprocess.call(["which", "x86_64-linux-gnu-gcc-13"], stdout=subprocess.DEVNULL) == 0 else "gcc"
        subprocess.check_call([cc, "-I", os.path.join(ROOT, "include"), src, "-o", exe])
        out = subprocess.check_output([exe]).decode().split()
    got = [int(v) for v in out]
    want = [C.sizeof(_abi.AbdParams), C.sizeof(_abi.AbdSceneDesc), C.sizeof(_abi.AbdStepStats),
            _abi.AbdParams.lin_tol.offset, _abi.AbdParams.precision.offset, _abi.AbdParams.pinned_diag.offset,
            _abi.AbdParams.warm_start.offset, _abi.AbdSceneDesc.planes.offset, _abi.AbdStepStats.gpu_ms.offset,
            _abi.AbdParams.ccd_max_iter.offset, _abi.AbdParams.test_inject.offset,
            _abi.AbdStepStats.solver_capped.offset, _abi.AbdStepStats.host_syncs.offset]
    assert got == want
