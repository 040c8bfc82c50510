"""Bloch phases of periodic structures on the GPU (tbgpu_set_bloch_k).

Bars: the reference's GaAs_bulk dense spectrum at all 40 k points within
2e-11 eV (the file prints 13 significant digits); H(k)*x against the oracle
within 45e-12 of max|H| on a strained periodic alloy supercell at an
arbitrary k; Hermiticity of H(k) to rounding; the Si_Bulk Lanczos eigenvalue
sets of the reference (same states per k, within 1e-6 eV); the no-allocation
entry point with phases equal to the regular one.
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu


def _dense(g):
    n = g.n
    h = np.zeros((n, n), complex)
    for c in range(n):
        x = np.zeros(2 * n)
        x[2 * c] = 1.0
        y = g.matvect_mult(x)
        h[:, c] = y[0::2] + 1j * y[1::2]
    return h


def _supercell(seed=5):
    rng = np.random.default_rng(seed)
    nx, ny, nz = 3, 2, 2
    t = np.zeros((nx, ny, nz, 8), np.uint8)
    t[..., :4] = np.where(rng.random((nx, ny, nz, 4)) < 0.5, materials.SPECIES["In"],
                          materials.SPECIES["Ga"])
    t[..., 4:] = materials.SPECIES["As"]
    dsp = rng.normal(0, 0.004, (nx, ny, nz, 8, 3))
    a = workloads.A_GAAS
    return workloads.Structure(nx, ny, nz, (a, a, a), (True, True, True), t, dsp)


def test_gaas_bulk_golden_all_k(golden):
    from nemo3d_b200.tbgpu import Hamiltonian
    ref = golden["gaas_bulk_kE"]
    st = workloads.bulk_cell("Ga", "As", 0.56532)
    g = Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS["GaAs_spds"]])
    worst = 0.0
    for kx in np.unique(ref[:, 0]):
        g.set_bloch_k([kx, 0.0, 0.0])
        h = _dense(g)
        assert np.abs(h - h.conj().T).max() <= 1e-13 * np.abs(h).max(), kx
        w = np.linalg.eigvalsh(h)
        want = np.sort(ref[ref[:, 0] == kx, 3])
        worst = max(worst, np.abs(w - want).max())
    assert worst < 2e-11, worst


@pytest.mark.parametrize("model", ["sp3d5s*_so", "sp3s*", "sp3s*_so"])
@pytest.mark.parametrize("variant", [0, 1])
def test_bloch_hx_matches_oracle(model, variant):
    from nemo3d_b200.tbgpu import Hamiltonian
    st = _supercell()
    fam = "spds" if model.startswith("sp3d5s") else "sps"
    mats = [materials.MATERIALS[f"GaAs_{fam}"], materials.MATERIALS[f"InAs_{fam}"]]
    norb, nspin = materials.BAND_MODELS[model]
    k = [0.31, -0.72, 0.45]
    g = Hamiltonian(st, model, mats)
    g.set_spmv_variant(variant)
    g.set_bloch_k(k)
    o = oracle.OracleHamiltonian(st, norb, nspin, mats, kvec=k)
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    for seed in (1, 2):
        x = workloads.random_start(g.n, seed=seed)
        y, yo = g.matvect_mult(x, shift=0.25), o.hx(x, shift=0.25)
        assert np.abs(y - yo).max() <= 45e-12 * scale
    # back to Gamma: no phases again
    g.set_bloch_k(None)
    o0 = oracle.OracleHamiltonian(st, norb, nspin, mats)
    x = workloads.random_start(g.n, seed=3)
    assert np.abs(g.matvect_mult(x) - o0.hx(x)).max() <= 45e-12 * scale


def test_si_bulk_lanczos_sets_on_gpu(golden):
    from nemo3d_b200.tbgpu import Hamiltonian
    ref = golden["si_bulk_kE"]
    st = workloads.bulk_cell("Si", "Si", 0.543095)
    g = Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS["Si_spds"]])
    cyc = [1.2, 0.8, -1.4, 0.1, -0.9, -0.2, 0.6]   # Lanczos.CyclicString
    r0 = np.array([cyc[i % 7] for i in range(2 * g.n)])
    for kx in np.unique(ref[:, 0])[::7]:
        g.set_bloch_k([kx, 0.0, 0.0])
        res = g.eigensolve_lanczos(r0, ConvCheckStartIter=200, ConvCheckSkipRate=50,
                                   imax=1000, requested1=20, requested2=20, emin1=-3,
                                   emax1=0.6, emin2=0.9, emax2=4, tolerance=1e-7)
        got = np.sort(res["values"])
        want = np.unique(ref[ref[:, 0] == kx, 3])
        assert len(got) == len(want), (kx, got, want)
        assert np.abs(got - want).max() < 1e-6, kx


def test_noalloc_with_phases_matches_regular_entry_point():
    import ctypes as C
    import torch
    from nemo3d_b200 import tbgpu
    st = _supercell(seed=9)
    mats = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]
    g = tbgpu.Hamiltonian(st, "sp3d5s*_so", mats)
    g.set_bloch_k([0.5, 0.25, -0.3])
    L = tbgpu._lib()
    L.tbgpu_hx_dot_noalloc.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    x = torch.from_numpy(workloads.random_start(g.n, seed=4)).cuda()
    y0, y1 = torch.empty_like(x), torch.empty_like(x)
    dot = torch.zeros(1, dtype=torch.float64, device="cuda")
    g.hx_dev(x.data_ptr(), y0.data_ptr(), shift=0.1)
    for _ in range(2):
        rc = L.tbgpu_hx_dot_noalloc(g._ctx, 0.1, C.c_void_p(x.data_ptr()),
                                    C.c_void_p(y1.data_ptr()), C.c_void_p(dot.data_ptr()))
        assert rc == 0
        torch.cuda.synchronize()
        assert (y1 - y0).abs().max().item() <= 1e-12 * y0.abs().max().item()
        assert abs(dot.item() - torch.dot(x, y1).item()) <= 1e-12 * abs(dot.item())
