"""GPU parity: libtbgpu.so (through its C ABI) against the CPU oracle.

Bars (stated per test):
* topology / neighbour lists / surface flags: bit-exact;
* Hamiltonian entries: |dH| <= 1e-12 * max|H| (the reference's FP64 code);
* H*x: |dy| <= 1e-12 * max|H| * max|x| * (number of couplings per row);
* Lanczos eigenvalues: same set as the oracle's run of the reference
  algorithm, each within 1e-6 eV.
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


def small_dome(seed=3):
    return workloads.dome_in_box(cells=(7, 6, 5), base_nm=2.4, height_nm=1.0,
                                 wl_z_nm=1.2, sigma_frac=0.02, seed=seed)


def pair(st, model, **kw):
    from nemo3d_b200.tbgpu import Hamiltonian
    mats = [materials.MATERIALS[m] for m in MODELS[model]]
    norb, nspin = materials.BAND_MODELS[model]
    g = Hamiltonian(st, model, mats, **kw)
    o = oracle.OracleHamiltonian(st, norb, nspin, mats, **kw)
    return g, o


@pytest.mark.parametrize("model", list(MODELS))
def test_pattern_bit_exact(model):
    st = small_dome()
    g, o = pair(st, model)
    site, nbr, surf = g.export_pattern()
    assert g.natoms == o.natoms
    np.testing.assert_array_equal(site, o.atom_slot)
    np.testing.assert_array_equal(nbr, o.nbr)
    np.testing.assert_array_equal(surf, o.surface)


@pytest.mark.parametrize("model", list(MODELS))
@pytest.mark.parametrize("strain", [True, False])
def test_hamiltonian_entries(model, strain):
    st = small_dome()
    g, o = pair(st, model, include_strain=strain)
    ons, blk = g.export_hamiltonian()
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    assert np.abs(ons - o.onsite).max() <= 1e-12 * scale
    assert np.abs(blk - o.blocks).max() <= 1e-12 * scale


@pytest.mark.parametrize("model", list(MODELS))
def test_hx_host_abi(model):
    st = small_dome()
    g, o = pair(st, model)
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, 2 * g.n)
    for shift in (0.0, 1.3):
        y = g.matvect_mult(x, shift)
        yo = o.hx(x, shift)
        scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
        assert np.abs(y - yo).max() <= 1e-12 * scale * 45


def test_hx_device_abi():
    import torch
    st = small_dome()
    g, o = pair(st, "sp3d5s*_so")
    x = torch.rand(2 * g.n, dtype=torch.float64, device="cuda") - 0.5
    y = torch.empty_like(x)
    g.hx_dev(x.data_ptr(), y.data_ptr(), 0.25)
    torch.cuda.synchronize()
    yo = o.hx(x.cpu().numpy(), 0.25)
    assert np.abs(y.cpu().numpy() - yo).max() <= 1e-10


def test_closed_cube_unbonded_and_surface():
    st = workloads.gaas_cube(3)
    st.types[0, 0, 0, 1] = 0          # site 5 of cell (0,0,0) loses its only bond
    g, o = pair(st, "sp3s*")
    site, nbr, surf = g.export_pattern()
    np.testing.assert_array_equal(site, o.atom_slot)
    np.testing.assert_array_equal(nbr, o.nbr)
    np.testing.assert_array_equal(surf, o.surface)


def test_gamma_point_golden(golden):
    """Periodic GaAs cell at k=0 on the GPU vs the reference's golden spectrum."""
    ref = golden["gaas_bulk_kE"]
    st = workloads.bulk_cell("Ga", "As", 0.56532)
    from nemo3d_b200.tbgpu import Hamiltonian
    g = Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS["GaAs_spds"]])
    n = g.n
    h = np.zeros((n, n), complex)
    for c in range(n):
        x = np.zeros(2 * n)
        x[2 * c] = 1.0
        y = g.matvect_mult(x)
        h[:, c] = y[0::2] + 1j * y[1::2]
    w = np.linalg.eigvalsh(h)
    want = np.sort(ref[ref[:, 0] == 0.0, 3])
    assert np.abs(w - want).max() < 2e-11


def _cube8_case():
    st = workloads.gaas_cube(8)
    return st, dict(requested1=4, requested2=3, emin1=-0.35, emax1=-0.25,
                    emin2=1.6, emax2=1.89, tolerance=1e-7, imax=4000,
                    ConvCheckStartIter=200, ConvCheckSkipRate=50)


def test_lanczos_cube8_eigenvalues_match_oracle():
    st, kw = _cube8_case()
    g, o = pair(st, "sp3s*")
    r0 = workloads.random_start(g.n, seed=0)
    res = g.eigensolve_lanczos(r0, **kw)
    ref = o.lanczos(r0, imax=kw["imax"], req=(kw["requested1"], kw["requested2"]),
                    erange1=(kw["emin1"], kw["emax1"]), erange2=(kw["emin2"], kw["emax2"]),
                    tol=kw["tolerance"], conv_start=200, conv_skip=50)
    assert len(res["values"]) == len(ref["evals"]) >= 7
    assert np.abs(np.sort(res["values"]) - np.sort(ref["evals"])).max() < 1e-6
    # the recurrence itself agrees (only summation order differs)
    # (rounding differences grow along the recurrence as orthogonality is lost)
    a, b = g.tridiagonal()
    assert np.abs(a[:30] - ref["alpha"][:30]).max() < 1e-11
    assert np.abs(a[:150] - ref["alpha"][:150]).max() < 1e-7


def test_lanczos_eigenvectors_and_determinism():
    st, kw = _cube8_case()
    g, o = pair(st, "sp3s*")
    r0 = workloads.random_start(g.n, seed=0)
    r1 = g.eigensolve_lanczos(r0, vectors=8, **kw)
    a1, b1 = g.tridiagonal()
    r2 = g.eigensolve_lanczos(r0, **kw)
    a2, b2 = g.tridiagonal()
    np.testing.assert_array_equal(a1, a2)          # deterministic reductions
    np.testing.assert_array_equal(b1, b2)
    np.testing.assert_array_equal(r1["values"], r2["values"])
    for lam, v in zip(r1["values"], r1["vectors"]):
        x = np.empty(2 * g.n)
        x[0::2], x[1::2] = v.real, v.imag
        hv = o.hx(x)
        hv = hv[0::2] + 1j * hv[1::2]
        nv = np.linalg.norm(v)
        assert abs(nv - 1.0) < 1e-3
        assert np.linalg.norm(hv - lam * v) / nv < 1e-4


def test_errors_are_codes_not_aborts():
    from nemo3d_b200 import tbgpu
    from nemo3d_b200.tbgpu import Hamiltonian, TbgpuError
    st = small_dome()
    with pytest.raises(TbgpuError) as e:   # no InAs parameter set given
        Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS["GaAs_spds"]])
    assert e.value.code == -4
    mats = [materials.MATERIALS[m] for m in MODELS["sp3d5s*_so"]]
    import torch
    g = Hamiltonian(st, "sp3d5s*_so", mats, build=False)
    bound = 2 * st.nsites * 20                 # >= 2 * dimension
    xd = torch.zeros(bound, dtype=torch.float64, device="cuda")
    yd = torch.zeros_like(xd)
    # rejected on the host (H not built yet) before any kernel is launched
    assert tbgpu._lib().tbgpu_hx_dev(g._ctx, 0.0, xd.data_ptr(), yd.data_ptr()) == -5
    g.build()
    with pytest.raises(TbgpuError) as e:
        g.build()                           # second build is out of order
    assert e.value.code == -5
    with pytest.raises(ValueError):
        g.matvect_mult(np.zeros(6))


def test_full_size_hermitian_and_linear():
    """1.02M-atom dome (58 x 58 x 38 cells): size-independent properties of H."""
    import torch
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.dome_in_box()
    g = Hamiltonian(st, "sp3d5s*_so",
                    [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]])
    assert g.natoms == 1022656
    gen = torch.Generator(device="cuda").manual_seed(5)
    u = torch.rand(2 * g.n, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    v = torch.rand(2 * g.n, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    hu, hv, hw = torch.empty_like(u), torch.empty_like(u), torch.empty_like(u)
    g.hx_dev(u.data_ptr(), hu.data_ptr())
    g.hx_dev(v.data_ptr(), hv.data_ptr())
    w = 0.3 * u - 1.7 * v
    g.hx_dev(w.data_ptr(), hw.data_ptr())
    torch.cuda.synchronize()
    cu = torch.view_as_complex(u.view(-1, 2))
    cv = torch.view_as_complex(v.view(-1, 2))
    chu = torch.view_as_complex(hu.view(-1, 2))
    chv = torch.view_as_complex(hv.view(-1, 2))
    lhs = torch.vdot(cu, chv)
    rhs = torch.vdot(chu, cv)
    assert abs(lhs - rhs).item() <= 1e-10 * abs(lhs).item() + 1e-8
    lin = hw - (0.3 * hu - 1.7 * hv)
    assert lin.abs().max().item() <= 1e-11 * hu.abs().max().item()


@pytest.mark.parametrize("model", ["sp3d5s*", "sp3d5s*_so"])
def test_spmv_variants_match_oracle(model):
    """Every H*x variant (warp-staged default, lane-gather, two-stage
    warp-staged, two-cell units) reproduces the oracle's H*x."""
    st = small_dome(seed=11)
    g, o = pair(st, model)
    x = np.random.default_rng(3).uniform(-1, 1, 2 * g.n)
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    yo = o.hx(x, 0.7)
    for variant in (0, 1, 2, 3, 4):
        g.set_spmv_variant(variant)
        assert np.abs(g.matvect_mult(x, 0.7) - yo).max() <= 1e-12 * scale * 45, variant


def test_lanczos_sp3d5s_so_dome_matches_oracle():
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    g, o = pair(st, "sp3d5s*_so")
    r0 = workloads.random_start(g.n, seed=0)
    kw = dict(imax=3000, requested1=3, requested2=3, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.4, tolerance=1e-7)
    res = g.eigensolve_lanczos(r0, **kw)
    ref = o.lanczos(r0, imax=3000, req=(3, 3), erange1=(-0.6, 0.3), erange2=(0.8, 2.4),
                    tol=1e-7)
    assert len(res["values"]) == len(ref["evals"]) >= 2
    assert np.abs(np.sort(res["values"]) - np.sort(ref["evals"])).max() < 1e-6


def test_cube8_eigenvalues_nearest_sigma():
    """The CPU-runnable case as stated: GaAs cube of 8x8x8 cells (4096 atoms),
    sp3s*, +30 eV passivation, start vector uniform in [-1, 1] from seed 0,
    the 8 eigenvalues nearest sigma = 1.6 eV.  Windows (sigma - 0.33, sigma]
    and (sigma, sigma + 0.33] with 8 requested in each run the solve to its
    iteration limit (the first window lies in the gap).  The 8 nearest
    eigenvalues with multiplicity come from LAPACK on the oracle's dense H
    (tests/golden/cube8_sp3s_dense.npz); single-vector Lanczos returns each
    degenerate level once, so the bar is: every distinct level among those 8
    is found, within 1e-6 eV, every value found is a dense eigenvalue
    within 1e-6 eV, and the GPU set equals the oracle's run."""
    import os
    sigma = 1.6
    dense = np.load(os.path.join(os.path.dirname(__file__), "golden", "cube8_sp3s_dense.npz"))
    w = dense["eigenvalues"]
    near8 = w[np.argsort(np.abs(w - sigma), kind="stable")[:8]]
    st = workloads.gaas_cube(8)
    g, o = pair(st, "sp3s*")
    assert g.natoms == int(dense["natoms"]) == 4096
    kw = dict(requested1=8, requested2=8, emin1=sigma - 0.33, emax1=sigma, emin2=sigma,
              emax2=sigma + 0.33, tolerance=1e-7, imax=6000, ConvCheckStartIter=200,
              ConvCheckSkipRate=50)
    r0 = workloads.random_start(g.n, seed=0)
    res = g.eigensolve_lanczos(r0, **kw)
    found = np.sort(res["values"])
    for lev in np.unique(np.round(near8, 9)):
        assert np.abs(found - lev).min() < 1e-6, (lev, found)
    for v in found:
        assert np.abs(w - v).min() < 1e-6, v
    ref = o.lanczos(r0, imax=kw["imax"], req=(8, 8), erange1=(kw["emin1"], kw["emax1"]),
                    erange2=(kw["emin2"], kw["emax2"]), tol=1e-7, conv_start=200, conv_skip=50)
    assert len(found) == len(ref["evals"])
    assert np.abs(found - np.sort(ref["evals"])).max() < 1e-6
    nearest = found[np.argsort(np.abs(found - sigma))[:8]]
    print("8 nearest distinct levels found:", np.round(np.sort(nearest), 9),
          "iterations", res["iterations"])
