"""Dense eigenvalues of the small CPU-runnable cube for the nearest-to-sigma parity case.

Workload: closed GaAs cube of 8 x 8 x 8 conventional cells (4096 atoms,
a = 0.56533 nm), sp3s* without spin-orbit (5 orbitals per atom, real H of
dimension 20480), dangling bonds passivated by +30 eV, no displacements.
The oracle assembles H (oracle/tb_oracle.c); LAPACK's dsyevr (through scipy)
returns every eigenvalue in (1.0, 2.3] eV with its multiplicity; those
below 2.0 eV are kept.  The GPU
test checks that the Lanczos solve for the 8 eigenvalues nearest 1.6 eV
returns the 8 nearest distinct values of this list.

Writes tests/golden/cube8_sp3s_dense.npz (under 2 kB).  Takes a few
minutes and ~12 GB of host memory.
"""
import os
import sys

import numpy as np
import scipy.linalg as sl

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from nemo3d_b200 import materials, workloads  # noqa: E402

WINDOW = (1.0, 2.3)
KEEP_BELOW = 2.0


def main():
    st = workloads.gaas_cube(8)
    mats = [materials.MATERIALS["GaAs_sps"], materials.MATERIALS["InAs_sps"]]
    o = oracle.OracleHamiltonian(st, 5, 1, mats)
    h = o.dense()
    assert np.abs(h.imag).max() == 0.0  # sp3s*, Gamma point: real symmetric
    hr = np.ascontiguousarray(h.real)
    del h
    w = sl.eigh(hr, eigvals_only=True, subset_by_value=WINDOW, driver="evr",
                overwrite_a=True, check_finite=False)
    w = np.sort(w)
    np.savez_compressed(os.path.join(HERE, "cube8_sp3s_dense.npz"), eigenvalues=w[w < KEEP_BELOW],
                        window=np.array([WINDOW[0], KEEP_BELOW]), natoms=o.natoms)
    print(o.natoms, "atoms;", len(w), "eigenvalues in", WINDOW, ":", np.round(np.sort(w), 6))


if __name__ == "__main__":
    main()
