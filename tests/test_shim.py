"""The eigensolve_lanczos drop-in compiled against the reference's own headers.

``tests/shim/build_shim.sh`` compiles nemo3d_b200/shim/eigensolve_lanczos_tbgpu.c
with the reference tree's eigen/include/lanczos.h in scope, so the compiler
checks the definition against the reference's declaration
(lanczos.h:365-391), and links it without undefined symbols to libtbgpu.so
and the test allocation stubs.  Bar: the build succeeds, warning-free for
the drop-in's own code, and the library exports ``eigensolve_lanczos``.
Skipped where the reference tree is absent and no build exists.
"""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SHIM = os.path.join(HERE, "shim", "_build", "libtbgpu_shim.so")
REF = os.environ.get("NEMO3D_SRC", "/root/reference/NEMO_3D")


def test_shim_compiles_against_reference_declaration():
    if os.path.isdir(REF):
        p = subprocess.run(["sh", os.path.join(HERE, "shim", "build_shim.sh"), REF],
                           capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        # no diagnostics from the drop-in itself (the nml headers' own
        # unused statics are silenced by the recipe)
        assert "eigensolve_lanczos_tbgpu.c" not in p.stderr, p.stderr
    if not os.path.exists(SHIM):
        pytest.skip("reference headers not present and no prebuilt shim")
    lib = ctypes.CDLL(SHIM)
    assert hasattr(lib, "eigensolve_lanczos")
    for name in ("nml_dv_new", "nml_dcv_new", "nml_dcm_new"):
        assert hasattr(lib, name)
