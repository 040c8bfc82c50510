"""The C ABI without a GPU: the library loads, exports every entry point that
include/tbgpu.h declares, runs its host-only functions like the oracle, and
fails loudly (an error code, no CPU fallback) when no CUDA device exists."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from nemo3d_b200 import build as nb
from nemo3d_b200 import materials, tbgpu, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tbgpu.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(tbgpu_[a-z_0-9]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    nb.build()
    return C.CDLL(nb.LIB)


def test_exports_every_declared_entry_point(lib):
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_error_strings(lib):
    lib.tbgpu_error_string.restype = C.c_char_p
    seen = set()
    for code in range(0, -9, -1):
        s = lib.tbgpu_error_string(code).decode()
        assert s and s not in seen
        seen.add(s)


@pytest.mark.parametrize("name", sorted(materials.MATERIALS))
@pytest.mark.parametrize("include_strain", [True, False])
def test_prepare_params_matches_oracle(name, include_strain):
    mat = materials.MATERIALS[name]
    ours = tbgpu.prepare_params(mat, include_strain)
    ref = oracle.prepare_params(mat, include_strain)
    assert np.array_equal(ours, ref)


def test_prepare_params_rejects_null(lib):
    lib.tbgpu_prepare_params.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_double, C.c_double, C.c_void_p]
    assert lib.tbgpu_prepare_params(0, 1, None, None, 0.0, 0.5, None) == -1


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    st = workloads.gaas_cube(2)
    with pytest.raises(tbgpu.TbgpuError) as e:
        tbgpu.Hamiltonian(st, "sp3s*")
    assert e.value.code in (-2, -3)  # TBGPU_E_CUDA / TBGPU_E_NOMEM
