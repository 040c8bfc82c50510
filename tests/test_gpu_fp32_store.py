"""Single-precision Hamiltonian store (tbgpu_set_ham_precision(32), the
reference's HamMemorySave build) on the GPU.

Bars: the exported store equals the oracle's FP64 entries rounded to float,
exactly; H*x equals the oracle's FP64 H*x over those rounded entries within
45e-12 of max|H| (the arithmetic stays double); against the FP64 store the
difference is float rounding (below 1e-6 of max|H|); Lanczos eigenvalues
move by less than 2e-5 eV from the FP64 store's (the error is printed per
state).
"""
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


def _rounded(o):
    r = oracle.OracleHamiltonian.__new__(oracle.OracleHamiltonian)
    r.__dict__.update(o.__dict__)
    r.onsite = o.onsite.astype(np.float32).astype(np.float64)
    r.blocks = o.blocks.astype(np.float32).astype(np.float64)
    return r


@pytest.mark.parametrize("model", list(MODELS))
@pytest.mark.parametrize("variant", [0, 1])
def test_fp32_store_hx(model, variant):
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _dome()
    mats = [materials.MATERIALS[m] for m in MODELS[model]]
    norb, nspin = materials.BAND_MODELS[model]
    g = Hamiltonian(st, model, mats, ham_bits=32)
    g.set_spmv_variant(variant)
    o = oracle.OracleHamiltonian(st, norb, nspin, mats)
    o32 = _rounded(o)
    ons, blk = g.export_hamiltonian()
    np.testing.assert_array_equal(ons, o32.onsite)
    np.testing.assert_array_equal(blk, o32.blocks)
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    for seed in (1, 2):
        x = workloads.random_start(g.n, seed=seed)
        y = g.matvect_mult(x, shift=0.2)
        assert np.abs(y - o32.hx(x, shift=0.2)).max() <= 45e-12 * scale
        assert np.abs(y - o.hx(x, shift=0.2)).max() <= 1e-6 * scale


def test_fp32_store_with_bloch_phases():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.bulk_cell("Ga", "As", 0.56532)
    mats = [materials.MATERIALS["GaAs_spds"]]
    g = Hamiltonian(st, "sp3d5s*_so", mats, ham_bits=32)
    k = [0.4, 0.0, 0.0]
    g.set_bloch_k(k)
    o32 = _rounded(oracle.OracleHamiltonian(st, 10, 2, mats, kvec=k))
    x = workloads.random_start(g.n, seed=7)
    scale = max(np.abs(o32.onsite).max(), np.abs(o32.blocks).max())
    assert np.abs(g.matvect_mult(x) - o32.hx(x)).max() <= 45e-12 * scale


def test_fp32_store_lanczos_error_per_state():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    mats = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]
    kw = dict(imax=5000, requested1=2, requested2=2, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.2, tolerance=1e-7)
    g64 = Hamiltonian(st, "sp3d5s*_so", mats)
    r0 = workloads.random_start(g64.n, seed=0)
    v64 = g64.eigensolve_lanczos(r0, **kw)["values"]
    v32 = Hamiltonian(st, "sp3d5s*_so", mats, ham_bits=32).eigensolve_lanczos(r0, **kw)["values"]
    assert len(v32) == len(v64) >= 4
    err = np.abs(np.sort(v32) - np.sort(v64))
    print("FP32 store eigenvalue error per state (eV):", err)
    assert err.max() < 2e-5


def test_precision_after_build_is_refused():
    from nemo3d_b200 import tbgpu
    g = tbgpu.Hamiltonian(workloads.gaas_cube(2), "sp3s*", [materials.MATERIALS["GaAs_sps"]])
    assert tbgpu._lib().tbgpu_set_ham_precision(g._ctx, 32) == -5
    assert tbgpu._lib().tbgpu_set_ham_precision(g._ctx, 16) == -1
