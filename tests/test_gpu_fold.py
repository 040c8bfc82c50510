"""Folded-spectrum operator (the reference's matvect_mult2) and the folded Lanczos solve.

Bars:
* F x = factor (H - s2)(H - s1) x + offset x through the matvect_mult2
  drop-in and the device entry point, against two oracle products:
  max |y - y_oracle| <= 1e-12 * max |y_oracle|, with the reference's
  constants (1.38, 1.58, -10, 0) and with other ones;
* folded Lanczos on a 288-site dot (dense diagonalisation possible): every
  returned value is an eigenvalue of F = f(lambda) of a dense eigenvalue
  lambda of H (within 1e-8 of |f|'s scale), the energies <v, H v> of the
  returned eigenvectors are those dense eigenvalues within 1e-6 eV, and the
  values of F found are the largest ones of its spectrum (the states nearest
  the fold's centre), each distinct level once.
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

MATS = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]


def _fold_oracle(o, x, s1, s2, factor, offset):
    t = o.hx(x, s1)
    return factor * o.hx(t, s2) + offset * x


@pytest.mark.parametrize("params", [(1.38, 1.58, -10.0, 0.0), (0.9, 1.7, 2.5, 0.75)])
def test_fold_product_matches_oracle(params):
    import torch
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.dome_in_box(cells=(7, 6, 5), base_nm=2.4, height_nm=1.0, wl_z_nm=1.2,
                               sigma_frac=0.02, seed=3)
    g = Hamiltonian(st, "sp3d5s*_so", MATS)
    o = oracle.OracleHamiltonian(st, 10, 2, MATS)
    g.set_fold(True, *params)
    x = workloads.random_start(g.n, seed=11)
    yo = _fold_oracle(o, x, *params)
    y = g.matvect_mult2(x)
    assert np.abs(y - yo).max() <= 1e-12 * np.abs(yo).max()
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    from nemo3d_b200 import tbgpu
    assert tbgpu._lib().tbgpu_hx_fold_dev(g._ctx, xd.data_ptr(), yd.data_ptr()) == 0
    torch.cuda.synchronize()
    assert np.abs(yd.cpu().numpy() - yo).max() <= 1e-12 * np.abs(yo).max()


def test_folded_lanczos_against_dense():
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.dome_in_box(cells=(3, 3, 4), base_nm=1.2, height_nm=0.6, wl_z_nm=0.6,
                               sigma_frac=0.01, seed=5)
    g = Hamiltonian(st, "sp3d5s*_so", MATS)
    o = oracle.OracleHamiltonian(st, 10, 2, MATS)
    lam = np.linalg.eigvalsh(o.dense())
    sigma, half = 1.3, 0.1
    s1, s2, factor = sigma - half, sigma + half, -10.0
    f = factor * (lam - s2) * (lam - s1)
    top = np.sort(f)[::-1]
    g.set_fold(True, s1, s2, factor, 0.0)
    # the window of F just below its largest values: the 3 highest distinct levels
    levels = np.unique(np.round(top, 7))[::-1]
    fmin = 0.5 * (levels[2] + levels[3])
    r0 = workloads.random_start(g.n, seed=0)
    res = g.eigensolve_lanczos(r0, ConvCheckStartIter=100, ConvCheckSkipRate=50, imax=8000,
                               requested1=0, requested2=3, emin1=0.0, emax1=0.0,
                               emin2=fmin, emax2=top[0] + 1.0, tolerance=1e-7, vectors=3)
    vals = np.sort(res["values"])[::-1]
    scale = np.abs(f).max()
    assert len(vals) == 3, (vals, levels[:4])
    for v in vals:
        assert np.abs(f - v).min() <= 1e-8 * scale, v
    np.testing.assert_allclose(vals, levels[:3], atol=1e-8 * scale)
    e = g.fold_energies()
    assert len(e) == 3
    for ei in e:
        assert np.abs(lam - ei).min() < 1e-6, ei
    # the energies are the levels nearest the fold's centre
    near = np.unique(np.round(lam[np.argsort(np.abs(lam - sigma))][:8], 7))
    assert all(np.abs(near - ei).min() < 1e-6 for ei in e)
    print("folded values", vals, "energies", np.sort(e), "iterations", res["iterations"])
