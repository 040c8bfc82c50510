"""Pin the CPU oracle to the reference's own golden data (no GPU needed).

* GaAs_bulk.old_nd_Ek_ascii: sp3d5s*+SO GaAs, one periodic cubic cell, 40 k
  points Gamma->X, all 160 eigenvalues per k by dense diagonalisation
  (ResFind=Direct, HamCompute=Recompute).  Pins Slater-Koster blocks,
  spin-orbit, on-site terms and Bloch phases.  Tolerance 2e-11 eV: the file
  prints 13 significant digits.
* Si_Bulk.old_nd_Ek_ascii: sp3d5s*+SO Si, Lanczos (SparseStore), windows
  [-3,0.6] and [0.9,4], 20+20 requested, tol 1e-7, CyclicRandom start.  Pins
  the Lanczos driver: the same eigenvalue *set* per k (which states converge
  and which are dropped as ghosts/degenerate), within 1e-6 eV.
* Si_Bulk.nd_nbrIndx: the 8x4 neighbour table of the periodic cell.
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads


def test_neighbour_table_matches_reference(golden):
    st = workloads.bulk_cell("Si", "Si", 0.543095)
    H = oracle.OracleHamiltonian(st, 10, 2, [materials.MATERIALS["Si_spds"]])
    assert H.natoms == 8
    np.testing.assert_array_equal(H.nbr.reshape(8, 4), golden["si_bulk_nbr"])


def test_gaas_bulk_dense_spectrum(golden):
    ref = golden["gaas_bulk_kE"]
    st = workloads.bulk_cell("Ga", "As", 0.56532)
    H = oracle.OracleHamiltonian(st, 10, 2, [materials.MATERIALS["GaAs_spds"]])
    for kx in np.unique(ref[:, 0]):
        h = H.dense([kx, 0.0, 0.0])
        assert np.abs(h - h.conj().T).max() == 0.0
        w = np.linalg.eigvalsh(h)
        g = np.sort(ref[ref[:, 0] == kx, 3])
        assert np.abs(w - g).max() < 2e-11, kx


@pytest.mark.parametrize("chunk", [0, 1, 2, 3])
def test_si_bulk_lanczos_sets(golden, chunk):
    ref = golden["si_bulk_kE"]
    ks = np.unique(ref[:, 0])[chunk::4]
    st = workloads.bulk_cell("Si", "Si", 0.543095)
    cyc = [1.2, 0.8, -1.4, 0.1, -0.9, -0.2, 0.6]   # Lanczos.CyclicString
    r0 = np.array([cyc[i % 7] for i in range(2 * 160)])
    for kx in ks:
        H = oracle.OracleHamiltonian(st, 10, 2, [materials.MATERIALS["Si_spds"]],
                                     kvec=[kx, 0, 0])
        res = H.lanczos(r0, imax=1000, req=(20, 20), erange1=(-3, 0.6),
                        erange2=(0.9, 4), tol=1e-7, conv_start=200, conv_skip=50)
        got = np.sort(res["evals"])
        want = np.unique(ref[ref[:, 0] == kx, 3])
        assert len(got) == len(want), (kx, got, want)
        assert np.abs(got - want).max() < 1e-6, (kx, got, want)


def test_cube8_dense_fixture_shape():
    """The dense fixture of the 4096-atom cube: sorted eigenvalues in the gap
    region's window, the conduction-band edge first (no level between 1.0 eV
    and it), and the multiplicities of the cube's symmetric states."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "cube8_sp3s_dense.npz"))
    w = d["eigenvalues"]
    assert int(d["natoms"]) == 4096
    assert np.all(np.diff(w) >= 0) and w[0] > 1.6 and w[-1] < 2.0
    assert abs(w[0] - 1.66814453) < 1e-7          # the conduction-band edge of the cube
    assert abs(w[1] - w[2]) < 1e-9                 # a doubly degenerate level next
