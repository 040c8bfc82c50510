"""The solver's per-device memory pool (tbgpu_release_solver_memory).

The Lanczos solves take their per-solve buffers from a pool that keeps its
memory mapped between solves.  Bars: two mixed-precision solves in a row with
the regenerating eigenvector pass (whose checkpoints come from the pool) give
the same values, iterations and eigenvectors bit for bit, with every
regenerated segment equal to its checkpoint; after the release the device's
free memory is larger by at least the checkpoints' size, and a third solve
still gives the same results.
"""
import numpy as np
import pytest

from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

MATS = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]
KW = dict(imax=4000, requested1=2, requested2=2, emin1=-0.6, emax1=0.3, emin2=0.8,
          emax2=2.6, tolerance=1e-7)


def test_pool_reuse_and_release():
    import torch
    from nemo3d_b200 import tbgpu
    st = workloads.dome_in_box(cells=(7, 6, 5), base_nm=2.4, height_nm=1.0, wl_z_nm=1.2,
                               sigma_frac=0.02, seed=3)
    g = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, ham_bits=32, lanczos_bits=32)
    g.set_spmv_variant(5)
    g.set_eigenvector_pass(1, 4, 64)
    r0 = workloads.random_start(g.n, seed=0)
    runs = []
    for k in range(2):
        res = g.eigensolve_lanczos(r0, vectors=4, **KW)
        s = g.stats()
        assert s["vec_segments"] >= 2 and s["vec_mismatch"] == 0, s
        runs.append(res)
    torch.cuda.synchronize()
    free_kept = torch.cuda.mem_get_info()[0]
    tbgpu.release_solver_memory()
    free_released = torch.cuda.mem_get_info()[0]
    # checkpoints: two complex-float vectors per 64 iterations
    ck = (runs[0]["iterations"] // 64) * 2 * g.n * 8
    print("free memory kept / released (MB):", free_kept / 2**20, free_released / 2**20,
          "checkpoints (MB):", ck / 2**20)
    assert free_released - free_kept >= ck
    runs.append(g.eigensolve_lanczos(r0, vectors=4, **KW))
    for r in runs[1:]:
        assert r["iterations"] == runs[0]["iterations"]
        np.testing.assert_array_equal(r["values"], runs[0]["values"])
        for a, b in zip(r["vectors"], runs[0]["vectors"]):
            np.testing.assert_array_equal(a, b)
