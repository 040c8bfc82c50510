"""Recomputed bond blocks (tbgpu_set_ham_storage(1), the reference's
HamCompute=Recompute): H*x evaluates every Slater-Koster block inside the
product instead of reading a stored one.

Bars: the blocks it works from equal the stored assembly's exactly; H*x
agrees with the stored path within 1e-13 and with the oracle within 45e-12 of
max|H| (four band models, strain, surfaces, Bloch phases); Lanczos finds the
same eigenvalues within 1e-9 eV.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

MODELS = {
    "sp3s*": ["GaAs_sps", "InAs_sps"],
    "sp3s*_so": ["GaAs_sps", "InAs_sps"],
    "sp3d5s*": ["GaAs_spds", "InAs_spds"],
    "sp3d5s*_so": ["GaAs_spds", "InAs_spds"],
}


def _dome(seed=3):
    return workloads.dome_in_box(cells=(7, 6, 5), base_nm=2.4, height_nm=1.0, wl_z_nm=1.2,
                                 sigma_frac=0.02, seed=seed)


@pytest.mark.parametrize("model", list(MODELS))
def test_recompute_hx(model):
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _dome()
    mats = [materials.MATERIALS[m] for m in MODELS[model]]
    norb, nspin = materials.BAND_MODELS[model]
    gs = Hamiltonian(st, model, mats)
    gr = Hamiltonian(st, model, mats, recompute=True)
    o = oracle.OracleHamiltonian(st, norb, nspin, mats)
    ons_s, blk_s = gs.export_hamiltonian()
    ons_r, blk_r = gr.export_hamiltonian()
    np.testing.assert_array_equal(ons_r, ons_s)
    np.testing.assert_array_equal(blk_r, blk_s)
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    for seed in (1, 2):
        x = workloads.random_start(gs.n, seed=seed)
        yr = gr.matvect_mult(x, shift=0.3)
        assert np.abs(yr - gs.matvect_mult(x, shift=0.3)).max() <= 1e-13 * scale
        assert np.abs(yr - o.hx(x, shift=0.3)).max() <= 45e-12 * scale


def test_recompute_with_bloch_phases():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.bulk_cell("Ga", "As", 0.56532)
    mats = [materials.MATERIALS["GaAs_spds"]]
    k = [0.35, 0.1, -0.2]
    g = Hamiltonian(st, "sp3d5s*_so", mats, recompute=True)
    g.set_bloch_k(k)
    o = oracle.OracleHamiltonian(st, 10, 2, mats, kvec=k)
    x = workloads.random_start(g.n, seed=4)
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    assert np.abs(g.matvect_mult(x) - o.hx(x)).max() <= 45e-12 * scale


def test_recompute_lanczos_matches_stored():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    mats = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]
    kw = dict(imax=1500, requested1=2, requested2=2, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.2, tolerance=1e-7)
    gs = Hamiltonian(st, "sp3d5s*_so", mats)
    r0 = workloads.random_start(gs.n, seed=0)
    vs = gs.eigensolve_lanczos(r0, **kw)["values"]
    vr = Hamiltonian(st, "sp3d5s*_so", mats, recompute=True).eigensolve_lanczos(r0, **kw)["values"]
    assert len(vs) == len(vr) > 0
    assert np.abs(vs - vr).max() < 1e-9


def test_recompute_refusals():
    import torch
    from nemo3d_b200 import tbgpu
    st = workloads.gaas_cube(2)
    with pytest.raises(tbgpu.TbgpuError) as e:
        tbgpu.Hamiltonian(st, "sp3d5s*", [materials.MATERIALS["GaAs_spds"]], recompute=True,
                          ham_bits=32)
    assert e.value.code == -6
    g = tbgpu.Hamiltonian(st, "sp3s*", [materials.MATERIALS["GaAs_sps"]], recompute=True)
    L = tbgpu._lib()
    L.tbgpu_hx_dot_noalloc.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    x = torch.zeros(2 * g.n, dtype=torch.float64, device="cuda")
    y, d = torch.empty_like(x), torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.tbgpu_hx_dot_noalloc(g._ctx, 0.0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                  C.c_void_p(d.data_ptr())) == -6
    assert L.tbgpu_set_ham_storage(g._ctx, 0) == -5
