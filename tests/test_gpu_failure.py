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


def test_batched_block_and_momentum_report_and_clear_status():
    """The batched, block and momentum entry points read the status word
    after their stream drains: after the self-test (status set, then cleared
    by its own report) each returns its normal result, the same as on a
    fresh context, and leaves the status clear for the next call."""
    from nemo3d_b200 import tbgpu
    mats = [materials.MATERIALS["GaAs_sps"], materials.MATERIALS["InAs_sps"]]
    dots = [workloads.alloy_dot(n, x, seed=i) for i, (n, x) in enumerate([(300, 0.5), (600, 0.8)])]
    packed, cells = workloads.pack_dots(dots)
    L = tbgpu._lib()
    L.tbgpu_selftest_bounded_wait.argtypes = [C.c_void_p, C.c_long]
    kw = dict(ConvCheckStartIter=100, ConvCheckSkipRate=50, imax=3000, requested1=1,
              requested2=2, tolerance=1e-7, emin1=-0.8, emax1=0.4, emin2=1.0, emax2=3.5)

    def batched(g):
        return g.eigensolve_lanczos_batched(workloads.random_start(g.n, seed=3), cells, **kw)

    g = tbgpu.Hamiltonian(packed, "sp3s*_so", mats)
    fresh = tbgpu.Hamiltonian(packed, "sp3s*_so", mats)
    assert L.tbgpu_selftest_bounded_wait(g._ctx, 4096) == TBGPU_E_TIMEOUT
    a, b = batched(g), batched(fresh)
    np.testing.assert_array_equal(a["iterations"], b["iterations"])
    for va, vb in zip(a["values"], b["values"]):
        np.testing.assert_array_equal(va, vb)
    x = workloads.random_start(g.n, seed=4)
    np.testing.assert_array_equal(g.matvect_mult(x), fresh.matvect_mult(x))
    assert L.tbgpu_last_error() == 0

    # block Lanczos and the momentum matrix on one dot
    d = tbgpu.Hamiltonian(dots[1], "sp3s*_so", mats)
    d2 = tbgpu.Hamiltonian(dots[1], "sp3s*_so", mats)
    assert L.tbgpu_selftest_bounded_wait(d._ctx, 4096) == TBGPU_E_TIMEOUT
    rb = np.stack([workloads.random_start(d.n, seed=20 + i) for i in range(2)])
    bk = dict(ConvCheckStartIter=50, ConvCheckSkipRate=25, imax=1500, requested1=1,
              requested2=1, emin1=-0.8, emax1=0.4, emin2=1.0, emax2=3.5, vectors=2)
    r1, r2 = d.eigensolve_blk_lanczos(rb, **bk), d2.eigensolve_blk_lanczos(rb, **bk)
    np.testing.assert_array_equal(r1["values"], r2["values"])
    assert L.tbgpu_selftest_bounded_wait(d._ctx, 4096) == TBGPU_E_TIMEOUT
    P1, _ = d.momentum_matrix(r1["vectors"])
    P2, _ = d2.momentum_matrix(r1["vectors"])
    np.testing.assert_array_equal(P1, P2)
    # the status word is clear: the next synchronous call reports success
    x1 = workloads.random_start(d.n, seed=5)
    np.testing.assert_array_equal(d.matvect_mult(x1), d2.matvect_mult(x1))
    assert L.tbgpu_last_error() == 0
