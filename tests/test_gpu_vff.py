"""Keating valence-force-field strain on the GPU (tbgpu_vff_energy,
tbgpu_vff_relax) against the oracle's restatement of calc_estrain and
macoptII_par.

Bars: energy within 1e-12 relative and gradient within 1e-12 of its largest
component at random displacements; the relaxation (same macopt algorithm)
ends at the oracle's displacements within 1e-7 nm and its energy within 1e-9
relative, for three boundary conditions; a Hamiltonian built after the
relaxation equals the oracle's Hamiltonian on the relaxed displacements
(H*x within 45e-12 of max|H|); refusals after the build and for a pair
without constants.
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

SPDS = ["GaAs_spds", "InAs_spds"]


def _dot(dsp_sigma=0.0):
    st = workloads.dome_in_box(cells=(6, 6, 5), base_nm=2.2, height_nm=1.0, wl_z_nm=0.6,
                               sigma_frac=0.0, seed=1)
    if dsp_sigma:
        rng = np.random.default_rng(7)
        st.dsp = rng.normal(0, dsp_sigma, (st.nx, st.ny, st.nz, 8, 3))
    return st


def test_energy_and_gradient_match_oracle():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _dot(dsp_sigma=0.003)
    vff = materials.vff_table()
    g = Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS[m] for m in SPDS], build=False)
    e, grad = g.vff_energy(vff, grad=True)
    o = oracle.OracleVFF(st, vff)
    eo, go = o.energy(o.from_sites(st.dsp))
    assert abs(e - eo) <= 1e-12 * abs(eo)
    go_sites = o.to_sites(go)
    assert np.abs(grad - go_sites).max() <= 1e-12 * np.abs(go).max()


@pytest.mark.parametrize("bc", [0, 2, 3])
def test_relaxation_matches_oracle(bc):
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _dot()
    vff = materials.vff_table()
    mats = [materials.MATERIALS[m] for m in SPDS]
    g = Hamiltonian(st, "sp3d5s*_so", mats, build=False)
    dsp, e, its = g.vff_relax(vff, bc=bc, max_iter=4000, tol=1e-10)
    o = oracle.OracleVFF(st, vff)
    uo, eo, itso = o.relax(bc=bc, itmax=4000, tol=1e-10)
    print(f"bc {bc}: GPU {its} iterations E {e:.12g}; oracle {itso} iterations E {eo:.12g}")
    assert abs(e - eo) <= 1e-9 * abs(eo)
    assert np.abs(o.from_sites(dsp) - uo).max() <= 1e-7
    # the build uses the relaxed displacements
    g.build()
    st.dsp = dsp
    oh = oracle.OracleHamiltonian(st, 10, 2, mats)
    x = workloads.random_start(g.n, seed=2)
    scale = max(np.abs(oh.onsite).max(), np.abs(oh.blocks).max())
    assert np.abs(g.matvect_mult(x) - oh.hx(x)).max() <= 45e-12 * scale


def test_vff_refusals():
    from nemo3d_b200 import tbgpu
    st = _dot()
    mats = [materials.MATERIALS[m] for m in SPDS]
    g = tbgpu.Hamiltonian(st, "sp3d5s*_so", mats)
    with pytest.raises(tbgpu.TbgpuError) as e:  # after the build
        g.vff_relax()
    assert e.value.code == -5
    g2 = tbgpu.Hamiltonian(st, "sp3d5s*_so", mats, build=False)
    with pytest.raises(tbgpu.TbgpuError) as e:  # no constants for InAs
        g2.vff_energy(materials.vff_table([("Ga", "As")]))
    assert e.value.code == -4
