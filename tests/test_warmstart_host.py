"""Host logic of the learned warm start (nemo3d_b200/warmstart.py), on CPU.

Bars: band-edge selection picks the 4 highest levels at or below sigma and
the 4 lowest above, or nothing when a side has fewer than 4; the search
windows sit on both sides of sigma; training targets from synthetic
eigenvectors have unit total probability per state (envelopes squared sum
to env_scale^2), each atom's probability lands in its voxel, and the
orbital profiles sum to 1 per state with both spins alike.
"""
import numpy as np
import pytest

from nemo3d_b200 import warmstart as ws
from nemo3d_b200 import workloads


def test_band_edges():
    v = np.array([0.1, 0.5, 0.6, 0.7, 0.8, 1.6, 1.7, 1.8, 1.9, 2.0])
    idx = ws.band_edges(v, 1.2)
    assert list(v[idx]) == [0.5, 0.6, 0.7, 0.8, 1.6, 1.7, 1.8, 1.9]
    assert ws.band_edges(v[:4], 1.2) is None          # no electrons
    assert ws.band_edges(v[2:8], 1.2) is None         # three holes
    assert list(ws.band_edges(v, 0.8)) == [1, 2, 3, 4, 5, 6, 7, 8]  # sigma on a level: a hole


def test_windows_straddle_sigma():
    kw = ws.solve_kw(1.1)
    assert kw["emin1"] < kw["emax1"] == 1.1 == kw["emin2"] < kw["emax2"]
    assert kw["requested1"] == kw["requested2"] == 4


class _FakeH:
    def __init__(self, st, site, nb):
        self.structure, self._site, self.nb = st, site, nb

    def export_pattern(self):
        return self._site, None, None


def test_targets_from_synthetic_vectors():
    st = workloads.lens_dot((4, 3, 2), base_nm=1.0, height_nm=0.5, x_in=0.5, seed=1)
    nb, G = 20, 2
    site = np.arange(st.nsites)  # every site an atom, in site order
    rng = np.random.default_rng(3)
    vec = rng.normal(size=(8, site.size * nb)) + 1j * rng.normal(size=(8, site.size * nb))
    values = np.array([0.5, 0.6, 0.7, 0.8, 1.6, 1.7, 1.8, 1.9])
    env, sigma, prof = ws.targets(_FakeH(st, site, nb), values, vec, G)
    assert sigma == pytest.approx(1.2)
    assert np.allclose((env ** 2).sum(1), ws.env_scale(G) ** 2)
    assert np.allclose(prof.sum((1, 2)), 1.0)
    assert np.allclose(prof[..., :10], prof[..., 10:])   # both spins alike
    # one state's probability per voxel, by hand
    p = (np.abs(vec[0].reshape(-1, nb)) ** 2).sum(1)
    p /= p.sum()
    cell = site >> 3
    k, j, i = cell % st.nz, (cell // st.nz) % st.ny, cell // (st.nz * st.ny)
    vox = ((i * G) // st.nx * G + (j * G) // st.ny) * G + (k * G) // st.nz
    want = np.sqrt(np.bincount(vox, p, G ** 3)) * ws.env_scale(G)
    assert np.allclose(env[0], want)
