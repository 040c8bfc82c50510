"""Momentum (optical) matrix elements on the GPU (tbgpu_momentum_matrix).

Oracle: ``oracle.momentum_matrix``, a literal restatement of the reference's
MOMENTUM_MATRIX block (eigsys3d_par.c:410-640: four H*x per final state and
direction, temp1 = <a|x H b>, temp2 = <a|H x b>).  Bars: the pXmatrix blocks
for x, y, z (labels exactly, values within 1e-10 of their largest entry) on a
strained alloy dome, for random states and for Lanczos eigenstates with the
transition table; spin-less models are refused.
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

SPDS = ["GaAs_spds", "InAs_spds"]


def _dome():
    return workloads.dome_in_box(cells=(6, 5, 4), base_nm=2.0, height_nm=0.8, wl_z_nm=0.9,
                                 sigma_frac=0.02, seed=4)


def _check(P, Po):
    np.testing.assert_array_equal(P[:, :, 0::2], Po[:, :, 0::2])  # labels
    scale = np.abs(Po[:, :, 1::2]).max()
    assert np.abs(P[:, :, 1::2] - Po[:, :, 1::2]).max() <= 1e-10 * scale


@pytest.mark.parametrize("model", ["sp3d5s*_so", "sp3s*_so"])
def test_momentum_matrix_random_states(model):
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _dome()
    fam = SPDS if model.startswith("sp3d5s") else ["GaAs_sps", "InAs_sps"]
    mats = [materials.MATERIALS[m] for m in fam]
    norb, nspin = materials.BAND_MODELS[model]
    g = Hamiltonian(st, model, mats)
    o = oracle.OracleHamiltonian(st, norb, nspin, mats)
    rng = np.random.default_rng(11)
    psi = rng.normal(size=(3, g.n)) + 1j * rng.normal(size=(3, g.n))
    psi /= np.linalg.norm(psi, axis=1, keepdims=True)
    P, _ = g.momentum_matrix(psi)
    Po, _ = oracle.momentum_matrix(o, psi)
    _check(P, Po)


def test_momentum_matrix_of_eigenstates_and_transitions():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _dome()
    mats = [materials.MATERIALS[m] for m in SPDS]
    g = Hamiltonian(st, "sp3d5s*_so", mats)
    res = g.eigensolve_lanczos(workloads.random_start(g.n, seed=0), imax=4000, requested1=2,
                               requested2=2, emin1=-0.6, emax1=0.3, emin2=0.8, emax2=2.5,
                               tolerance=1e-7, vectors=4)
    psi, E = res["vectors"], res["values"][:4]
    assert len(psi) == 4
    P, T = g.momentum_matrix(psi, E)
    o = oracle.OracleHamiltonian(st, 10, 2, mats)
    Po, To = oracle.momentum_matrix(o, psi, E)
    _check(P, Po)
    np.testing.assert_array_equal(T[..., :3], To[..., :3])
    assert np.abs(T[..., 3] - To[..., 3]).max() <= 1e-9 * To[..., 3].max()


def test_momentum_matrix_refused_without_spin():
    from nemo3d_b200 import tbgpu
    g = tbgpu.Hamiltonian(workloads.gaas_cube(2), "sp3d5s*", [materials.MATERIALS["GaAs_spds"]])
    with pytest.raises(tbgpu.TbgpuError) as e:
        g.momentum_matrix(np.ones((1, g.n), complex))
    assert e.value.code == -6
