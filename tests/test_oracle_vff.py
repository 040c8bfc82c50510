"""The oracle's Keating valence-force-field restatement (CPU).

Bars: an unstrained binary at its own lattice constant has zero energy and
zero gradient, exactly; the gradient is the reference's, i.e. the exact
gradient of (bond stretching / 2 + bond bending), checked by central
differences; a relaxation lowers the energy, leaves the fixed atoms of every
boundary condition where they were and ends with a small gradient.
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads


def _dot(cells=(5, 5, 4)):
    return workloads.dome_in_box(cells=cells, base_nm=2.0, height_nm=0.9, wl_z_nm=0.6,
                                 sigma_frac=0.0, seed=1)


def test_unstrained_binary_has_zero_energy():
    o = oracle.OracleVFF(workloads.gaas_cube(3), materials.vff_table())
    e, g = o.energy(np.zeros((o.natoms, 3)))
    assert e == 0.0
    assert np.abs(g).max() == 0.0


def test_gradient_is_half_stretch_plus_bend():
    st = _dot()
    vff = materials.vff_table()
    o = oracle.OracleVFF(st, vff)
    vff2 = vff.copy()
    vff2[..., 1] *= 2  # doubles the stretching energy only
    o2 = oracle.OracleVFF(st, vff2)
    rng = np.random.default_rng(3)
    u = rng.normal(0, 0.003, (o.natoms, 3))
    _, g = o.energy(u)
    f = lambda v: 1.5 * o.energy(v)[0] - 0.5 * o2.energy(v)[0]  # stretch/2 + bend
    for k in range(3):
        d = rng.normal(size=u.shape)
        h = 1e-6
        fd = (f(u + h * d) - f(u - h * d)) / (2 * h)
        assert abs(fd - (g * d).sum()) <= 1e-6 * abs(fd)


@pytest.mark.parametrize("bc", [0, 1, 2, 3, 4])
def test_relaxation(bc):
    st = _dot()
    o = oracle.OracleVFF(st, materials.vff_table())
    e0, _ = o.energy(np.zeros((o.natoms, 3)))
    u, e, its = o.relax(bc=bc, itmax=4000, tol=1e-10)
    free = o.free_mask(bc)
    assert its < 4000
    assert e < e0
    assert np.abs(u[~free]).max(initial=0.0) == 0.0
    _, g = o.energy(u)
    assert np.abs(g[free]).max() < 1e-4 * np.abs(o.energy(np.zeros_like(u))[1]).max()
    if bc == 1:
        assert (~free).sum() == 1
    if bc == 3:
        k = (o.atom_slot // 8) % st.nz
        assert np.array_equal(~free, k <= 1)
