"""Eigenvector and eigenvalue files of a GPU solve in the reference's <HDR>
format, read back: the records equal the vectors and values the solver
returned, bit for bit; the header carries the basis size, atom count, band
model and crystal structure as the reference writes them."""
import numpy as np
import pytest

from nemo3d_b200 import materials, nd_files, workloads

pytestmark = pytest.mark.gpu


def test_solve_results_round_trip(tmp_path):
    from nemo3d_b200 import tbgpu
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    mats = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]
    g = tbgpu.Hamiltonian(st, "sp3d5s*_so", mats)
    r0 = workloads.random_start(g.n, seed=0)
    res = g.eigensolve_lanczos(r0, imax=1500, requested1=2, requested2=2, emin1=-0.6,
                               emax1=0.3, emin2=0.8, emax2=2.2, tolerance=1e-7, vectors=2)
    ek = str(tmp_path / "dot.nd_Ek")
    tbgpu.write_eigenvalues(ek, "i", None, [])
    tbgpu.write_eigenvalues(ek, "a", (0.0, 0.0, 0.0), res["values"])
    kE = nd_files.read_eigenvalues(ek)
    np.testing.assert_array_equal(kE[:, 3], res["values"])
    for i, v in enumerate(res["vectors"]):
        path = str(tmp_path / f"dot.nd_evec_{i + 1}")
        g.write_eigenvector(path, v)
        hdr, _ = nd_files.read(path)
        assert hdr["format"] == "{real wf.r, real wf.i}"
        assert hdr["dims"] == [20, g.natoms]
        assert hdr["user"][0] == "Bands_20_sp3d5ss_spin # band_model"
        assert hdr["user"][1] == "2 # crystal structure"
        np.testing.assert_array_equal(nd_files.read_eigenvector(path), v)
