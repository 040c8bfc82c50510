"""H*x variant 3 (two-cell units, bulk-copied) against the default kernel.

Bars: y bit-identical to variant 0 (same per-lane arithmetic in the same
order) on domes with surfaces and passivation, odd cell counts along z, a
periodic supercell at the Gamma point, both 10-orbital models, with and
without a shift; the fallback for other models equal too; unaligned vectors refused;
H*x against the oracle within 45e-12 of max|H|; Lanczos eigenvalues within
1e-9 eV of the default kernel's (alpha is summed in another order).
"""
import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu


def _ham(st, model, fam="spds"):
    from nemo3d_b200.tbgpu import Hamiltonian
    mats = [materials.MATERIALS[f"GaAs_{fam}"], materials.MATERIALS[f"InAs_{fam}"]]
    return Hamiltonian(st, model, mats), mats


def _supercell(seed=5):
    rng = np.random.default_rng(seed)
    nx, ny, nz = 3, 4, 3
    t = np.zeros((nx, ny, nz, 8), np.uint8)
    t[..., :4] = np.where(rng.random((nx, ny, nz, 4)) < 0.5, materials.SPECIES["In"],
                          materials.SPECIES["Ga"])
    t[..., 4:] = materials.SPECIES["As"]
    dsp = rng.normal(0, 0.004, (nx, ny, nz, 8, 3))
    a = workloads.A_GAAS
    return workloads.Structure(nx, ny, nz, (a, a, a), (True, True, True), t, dsp)


STRUCTURES = {
    "dome_7x6x5": lambda: workloads.dome_in_box(cells=(7, 6, 5), base_nm=2.4, height_nm=1.0,
                                                wl_z_nm=1.2, sigma_frac=0.02, seed=3),
    "dome_20x18x13": lambda: workloads.dome_in_box(cells=(20, 18, 13), base_nm=7.0,
                                                   height_nm=2.0, wl_z_nm=1.5,
                                                   sigma_frac=0.02, seed=4),
    "periodic_3x4x3": _supercell,
    "alloy_dot": lambda: workloads.alloy_dot(6000, 0.3, seed=2),
}


@pytest.mark.parametrize("name", list(STRUCTURES))
@pytest.mark.parametrize("model", ["sp3d5s*", "sp3d5s*_so"])
def test_tile_bit_identical(name, model):
    g, _ = _ham(STRUCTURES[name](), model)
    rng = np.random.default_rng(17)
    x = rng.uniform(-1, 1, 2 * g.n)
    for shift in (0.0, 0.9):
        g.set_spmv_variant(0)
        y0 = g.matvect_mult(x, shift)
        g.set_spmv_variant(3)
        y3 = g.matvect_mult(x, shift)
        np.testing.assert_array_equal(y3, y0)


def test_tile_matches_oracle():
    st = STRUCTURES["dome_7x6x5"]()
    g, mats = _ham(st, "sp3d5s*_so")
    o = oracle.OracleHamiltonian(st, 10, 2, mats)
    g.set_spmv_variant(3)
    x = np.random.default_rng(5).uniform(-1, 1, 2 * g.n)
    scale = max(np.abs(o.onsite).max(), np.abs(o.blocks).max())
    assert np.abs(g.matvect_mult(x, 0.4) - o.hx(x, 0.4)).max() <= 45e-12 * scale


def test_tile_device_pointers_and_unaligned_refusal():
    import torch
    from nemo3d_b200.tbgpu import TbgpuError
    g, _ = _ham(STRUCTURES["dome_20x18x13"](), "sp3d5s*_so")
    n2 = 2 * g.n
    x = torch.rand(n2, dtype=torch.float64, device="cuda") - 0.5
    y0, y3 = (torch.empty(n2, dtype=torch.float64, device="cuda") for _ in range(2))
    g.set_spmv_variant(0)
    g.hx_dev(x.data_ptr(), y0.data_ptr(), 0.3)
    g.set_spmv_variant(3)
    g.hx_dev(x.data_ptr(), y3.data_ptr(), 0.3)
    torch.cuda.synchronize()
    assert torch.equal(y3, y0)
    # a vector that does not start on a 16-byte boundary is refused before
    # any launch, whatever the variant
    base = torch.zeros(n2 + 2, dtype=torch.float64, device="cuda")
    for variant in (0, 3):
        g.set_spmv_variant(variant)
        with pytest.raises(TbgpuError):
            g.hx_dev(base.data_ptr() + 8, y0.data_ptr())
        with pytest.raises(TbgpuError):
            g.hx_dev(x.data_ptr(), base.data_ptr() + 8)


def test_tile_other_models_fall_back():
    g, _ = _ham(STRUCTURES["dome_7x6x5"](), "sp3s*_so", fam="sps")
    x = np.random.default_rng(9).uniform(-1, 1, 2 * g.n)
    g.set_spmv_variant(0)
    y0 = g.matvect_mult(x, 0.2)
    g.set_spmv_variant(3)
    np.testing.assert_array_equal(g.matvect_mult(x, 0.2), y0)


@pytest.mark.parametrize("name", list(STRUCTURES))
@pytest.mark.parametrize("model", ["sp3d5s*", "sp3d5s*_so"])
def test_bulk_block_runs_bit_identical(name, model):
    """Variant 0 (cation block runs by bulk copy) and variant 4 (by cp.async)
    stage the same bytes for the same arithmetic."""
    g, _ = _ham(STRUCTURES[name](), model)
    x = np.random.default_rng(23).uniform(-1, 1, 2 * g.n)
    for shift in (0.0, 0.6):
        g.set_spmv_variant(0)
        y0 = g.matvect_mult(x, shift)
        g.set_spmv_variant(4)
        np.testing.assert_array_equal(g.matvect_mult(x, shift), y0)


def test_bulk_lanczos_matches_default():
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    g, _ = _ham(st, "sp3d5s*_so")
    r0 = workloads.random_start(g.n, seed=0)
    kw = dict(imax=3000, requested1=3, requested2=3, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.4, tolerance=1e-7)
    g.set_spmv_variant(0)
    ref = g.eigensolve_lanczos(r0, **kw)
    g.set_spmv_variant(4)
    res = g.eigensolve_lanczos(r0, **kw)
    assert res["iterations"] == ref["iterations"]
    np.testing.assert_array_equal(res["values"], ref["values"])


def test_autotune_selects_a_variant_with_the_same_product():
    g, _ = _ham(STRUCTURES["dome_20x18x13"](), "sp3d5s*_so")
    x = np.random.default_rng(31).uniform(-1, 1, 2 * g.n)
    g.set_spmv_variant(0)
    y0 = g.matvect_mult(x, 0.3)
    v, ms = g.autotune_spmv(reps=5)
    assert v in (0, 1, 2, 3, 4, 5, 6, 8, 9) and ms > 0.0
    y = g.matvect_mult(x, 0.3)
    if v in (1, 5, 6, 8, 9):  # kernels that sum in their own orders
        ons, blk = g.export_hamiltonian()
        assert np.abs(y - y0).max() <= 1e-13 * max(np.abs(ons).max(), np.abs(blk).max())
    else:
        np.testing.assert_array_equal(y, y0)
    # a 5-orbital model: the lane-gather kernel at 8, 4 or 2 warps per block,
    # one product
    h, _ = _ham(STRUCTURES["dome_7x6x5"](), "sp3s*_so", fam="sps")
    h.set_spmv_variant(0)
    z0 = h.matvect_mult(x[:2 * h.n], 0.3)
    v, ms = h.autotune_spmv(reps=3)
    assert v in (0, 8, 9) and ms > 0.0
    np.testing.assert_array_equal(h.matvect_mult(x[:2 * h.n], 0.3), z0)


@pytest.mark.parametrize("model,fam,bloch", [("sp3s*_so", "sps", False), ("sp3s*", "sps", False),
                                             ("sp3d5s*_so", "spds", False),
                                             ("sp3d5s*_so", "spds", True)])
def test_lane_gather_block_sizes_same_product(model, fam, bloch):
    """Variants 1, 8 and 9 (the lane-gather kernel with 8, 4 and 2 warps per
    block) give y bit for bit, with and without Bloch phases; a Lanczos solve
    on variant 9 finds the values of variant 1 to 1e-9 eV (the fused alpha
    dot sums its block partials over another block count)."""
    g, _ = _ham(STRUCTURES["periodic_3x4x3" if bloch else "dome_7x6x5"](), model, fam=fam)
    if bloch:
        g.set_bloch_k([0.11, -0.07, 0.05])
    x = np.random.default_rng(5).uniform(-1, 1, 2 * g.n)
    ys = []
    for v in (1, 8, 9):
        g.set_spmv_variant(v)
        ys.append(g.matvect_mult(x, 0.2))
    np.testing.assert_array_equal(ys[0], ys[1])
    np.testing.assert_array_equal(ys[0], ys[2])
    if bloch:
        return
    r0 = workloads.random_start(g.n, seed=0)
    kw = dict(imax=3000, requested1=2, requested2=2, emin1=-0.6, emax1=0.4, emin2=1.0,
              emax2=2.6, tolerance=1e-7)
    g.set_spmv_variant(1)
    a = g.eigensolve_lanczos(r0, **kw)
    g.set_spmv_variant(9)
    b = g.eigensolve_lanczos(r0, **kw)
    assert len(a["values"]) > 0 and len(b["values"]) > 0
    for u, w in ((a["values"], b["values"]), (b["values"], a["values"])):
        assert max(np.abs(w - t).min() for t in u) < 1e-9


def test_tile_variant_range():
    from nemo3d_b200.tbgpu import TbgpuError
    g, _ = _ham(STRUCTURES["dome_7x6x5"](), "sp3d5s*")
    g.set_spmv_variant(7)  # the staged pencil kernel (the pencil kernel where it does not apply)
    g.set_spmv_variant(8)  # the lane-gather kernel with 4 and 2 warps per block
    g.set_spmv_variant(9)
    with pytest.raises(TbgpuError):
        g.set_spmv_variant(10)
    with pytest.raises(TbgpuError):
        g.set_spmv_variant(-1)


def test_tile_lanczos_matches_default():
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    g, _ = _ham(st, "sp3d5s*_so")
    r0 = workloads.random_start(g.n, seed=0)
    kw = dict(imax=3000, requested1=3, requested2=3, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.4, tolerance=1e-7)
    g.set_spmv_variant(0)
    ref = g.eigensolve_lanczos(r0, **kw)
    g.set_spmv_variant(3)
    res = g.eigensolve_lanczos(r0, **kw)
    assert len(res["values"]) == len(ref["values"]) >= 2
    assert np.abs(np.sort(res["values"]) - np.sort(ref["values"])).max() < 1e-9


def test_start_vector_seam_and_device_matvec():
    """tbgpu_set_start_vector: a solve without r_0 uses the stored vector
    (same result as passing it); tbgpu_matvect_mult_dev equals hx_dev."""
    import ctypes as C
    import torch
    from nemo3d_b200 import tbgpu
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    g, _ = _ham(st, "sp3d5s*_so")
    r0 = workloads.random_start(g.n, seed=4)
    kw = dict(imax=3000, requested1=2, requested2=2, emin1=-0.6, emax1=0.3, emin2=0.8,
              emax2=2.4, tolerance=1e-7)
    ref = g.eigensolve_lanczos(r0, **kw)
    g.set_start_vector(r0)
    res = g.eigensolve_lanczos(None, **kw)
    assert res["iterations"] == ref["iterations"]
    np.testing.assert_array_equal(res["values"], ref["values"])
    g.set_start_vector(None)
    with pytest.raises(tbgpu.TbgpuError):
        g.eigensolve_lanczos(None, **kw)
    x = torch.rand(2 * g.n, dtype=torch.float64, device="cuda") - 0.5
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    g.hx_dev(x.data_ptr(), y1.data_ptr(), 0.25)
    shift = C.c_double(0.25)
    args = (C.c_void_p * 3)(g._ctx.value, C.cast(C.pointer(shift), C.c_void_p).value, None)
    tbgpu._lib().tbgpu_matvect_mult_dev(args, C.c_void_p(y2.data_ptr()),
                                        C.c_void_p(x.data_ptr()))
    torch.cuda.synchronize()
    assert tbgpu._lib().tbgpu_last_error() == 0
    assert torch.equal(y1, y2)
