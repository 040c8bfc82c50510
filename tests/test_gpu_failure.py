"""Failure detection without a GPU fault.

Bar: a device-side wait on an mbarrier that nothing completes runs out
after its bounded poll count and reports TBGPU_E_TIMEOUT through the
context's status word (no trap, no hang); the status word is cleared on
report, and the same context then gives the same H*x and a normal solve.
"""
import ctypes as C

import numpy as np
import pytest

from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

TBGPU_E_TIMEOUT = -8


def test_bounded_wait_reports_timeout_and_context_survives():
    from nemo3d_b200 import tbgpu
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    g = tbgpu.Hamiltonian(st, "sp3d5s*_so",
                          [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]])
    x = workloads.random_start(g.n, seed=5)
    y0 = g.matvect_mult(x, 0.1)
    L = tbgpu._lib()
    L.tbgpu_selftest_bounded_wait.argtypes = [C.c_void_p, C.c_long]
    assert L.tbgpu_selftest_bounded_wait(g._ctx, 0) == -1          # bad poll count
    assert L.tbgpu_selftest_bounded_wait(g._ctx, 4096) == TBGPU_E_TIMEOUT
    assert L.tbgpu_last_error() == TBGPU_E_TIMEOUT
    np.testing.assert_array_equal(g.matvect_mult(x, 0.1), y0)     # status cleared, same product
    kw = dict(imax=1500, requested1=2, requested2=2, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.2, tolerance=1e-7)
    r0 = workloads.random_start(g.n, seed=0)
    res = g.eigensolve_lanczos(r0, **kw)  # raises if the status word were still set
    fresh = tbgpu.Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS["GaAs_spds"],
                                                 materials.MATERIALS["InAs_spds"]])
    ref = fresh.eigensolve_lanczos(r0, **kw)
    assert res["iterations"] == ref["iterations"]
    np.testing.assert_array_equal(res["values"], ref["values"])
