"""Tensor-core block dots (tbgpu_block_dots_dev, tcgen05.mma kind::i8 on
7-bit slices of the double entries) against numpy's double-precision X^H Y,
and block Lanczos with its dots on the tensor cores against the same solve on
the CUDA-core kernel.

Bars:
* |G_ij - (X^H Y)_ij| <= 1e-13 ||x_i|| ||y_j|| for p = 1..8, lengths that
  are and are not multiples of the 256-entry chunk, vectors whose scales
  differ by 10^12 and vectors with entries spread over 30 decades;
* small-integer entries give the exact integer products (every slice product
  and every double sum is exact);
* zero blocks give zero, X^H X is Hermitian to rounding with a positive
  diagonal;
* block Lanczos (the reference's eigensolve_blk_lanczos parameters) with
  tensor-core dots finds the same distinct values to 1e-9 eV as with the
  CUDA-core dots (counts per window may differ only by copies of an exactly
  degenerate value, which the reference's Method-4 test keeps or not
  depending on rounding), in the same number of block steps within one
  convergence check;
* invalid block sizes, lengths and misaligned pointers raise TBGPU_E_ARG.
"""
import numpy as np
import pytest

from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu


def _ham():
    from nemo3d_b200.tbgpu import Hamiltonian
    return Hamiltonian(workloads.gaas_cube(2), "sp3s*", [materials.MATERIALS["GaAs_sps"]])


def _dev(z):
    """complex (p, n) -> contiguous device doubles (p, 2n), interleaved"""
    import torch
    a = np.empty((z.shape[0], 2 * z.shape[1]))
    a[:, 0::2], a[:, 1::2] = z.real, z.imag
    return torch.from_numpy(a).cuda()


def _tc(g, X, Y):
    xd, yd = _dev(X), _dev(Y)
    G = g.block_dots_dev(X.shape[0], xd.data_ptr(), yd.data_ptr(), X.shape[1])
    return G


def _check(G, X, Y, rel=1e-13):
    ref = X.conj() @ Y.T
    bound = rel * np.outer(np.linalg.norm(X, axis=1), np.linalg.norm(Y, axis=1))
    err = np.abs(G - ref)
    print("max err / bound", (err / np.maximum(bound, 1e-300)).max())
    assert np.all(err <= bound), (err.max(), bound.min())


@pytest.mark.parametrize("p", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("n2", [1, 255, 256, 4097, 100003])
def test_block_dots_random(p, n2):
    g = _ham()
    rng = np.random.default_rng(p * 1000 + n2)
    X = rng.standard_normal((p, n2)) + 1j * rng.standard_normal((p, n2))
    Y = rng.standard_normal((p, n2)) + 1j * rng.standard_normal((p, n2))
    _check(_tc(g, X, Y), X, Y)


def test_block_dots_scales_and_dynamic_range():
    g = _ham()
    rng = np.random.default_rng(5)
    p, n2 = 8, 70001
    X = rng.standard_normal((p, n2)) + 1j * rng.standard_normal((p, n2))
    Y = rng.standard_normal((p, n2)) + 1j * rng.standard_normal((p, n2))
    X *= (10.0 ** np.arange(-6, 2))[:, None]            # vector scales 1e-6 .. 10
    Y *= 10.0 ** rng.uniform(-30, 0, size=(p, n2))      # entries over 30 decades
    Y[3] *= 1e6
    _check(_tc(g, X, Y), X, Y)
    # a localised vector: a few large entries, the rest tiny
    Z = Y.copy()
    Z[:, ::1000] *= 1e12
    _check(_tc(g, X, Z), X, Z)


def test_block_dots_exact_integers():
    g = _ham()
    rng = np.random.default_rng(9)
    p, n2 = 8, 30011
    Xi = rng.integers(-100, 101, size=(p, n2, 2))
    Yi = rng.integers(-100, 101, size=(p, n2, 2))
    X, Y = Xi[..., 0] + 1j * Xi[..., 1], Yi[..., 0] + 1j * Yi[..., 1]
    G = _tc(g, X, Y)
    rr = np.einsum("ik,jk->ij", Xi[..., 0], Yi[..., 0]) + np.einsum("ik,jk->ij", Xi[..., 1], Yi[..., 1])
    ri = np.einsum("ik,jk->ij", Xi[..., 0], Yi[..., 1]) - np.einsum("ik,jk->ij", Xi[..., 1], Yi[..., 0])
    np.testing.assert_array_equal(G.real, rr.astype(np.float64))
    np.testing.assert_array_equal(G.imag, ri.astype(np.float64))


def test_block_dots_zero_and_hermitian():
    g = _ham()
    p, n2 = 4, 5000
    Z = np.zeros((p, n2), complex)
    assert np.all(_tc(g, Z, Z) == 0.0)
    rng = np.random.default_rng(3)
    X = rng.standard_normal((p, n2)) + 1j * rng.standard_normal((p, n2))
    G = _tc(g, X, X)
    # re.im and im.re of one vector are summed in different orders: the
    # diagonal's imaginary part is rounding, as in a double dot with FMA
    assert np.all(np.abs(G.diagonal().imag) <= 1e-13 * G.diagonal().real)
    assert np.all(G.diagonal().real > 0.0)
    np.testing.assert_allclose(G, G.conj().T, rtol=0, atol=1e-13 * np.abs(G).max())
    _check(G, X, X)


def test_block_dots_argument_errors():
    import torch
    from nemo3d_b200.tbgpu import TbgpuError
    g = _ham()
    x = torch.zeros(8 * 2 * 64 + 2, dtype=torch.float64, device="cuda")
    for p, n2, off in ((0, 64, 0), (9, 64, 0), (2, 0, 0), (2, 64, 1)):
        with pytest.raises(TbgpuError) as e:
            g.block_dots_dev(p, x.data_ptr() + 8 * off, x.data_ptr(), n2)
        assert e.value.code == -1
    with pytest.raises(TbgpuError):
        g.set_block_dots(2)


@pytest.mark.parametrize("model,cube,p,skip", [("sp3d5s*_so", 2, 4, 10), ("sp3d5s*_so", 2, 8, 10),
                                               ("sp3s*", 3, 8, 10)])
def test_block_lanczos_tensor_dots(model, cube, p, skip):
    from nemo3d_b200.tbgpu import Hamiltonian
    fam = "spds" if model.startswith("sp3d5s") else "sps"
    st = workloads.gaas_cube(cube)
    g = Hamiltonian(st, model, [materials.MATERIALS[f"GaAs_{fam}"]])
    r0 = np.random.default_rng(11).uniform(-1, 1, size=(p, 2 * g.n))
    kw = dict(imax=min(300, g.n // p - 2), requested1=3, requested2=3, emin1=-1.5,
              emax1=0.5, emin2=1.0, emax2=3.5, tolerance=1e-7, ConvCheckStartIter=30,
              ConvCheckSkipRate=skip)
    g.set_block_dots(0)
    a = g.eigensolve_blk_lanczos(r0, **kw)
    g.set_block_dots(1)
    b = g.eigensolve_blk_lanczos(r0, **kw)
    g.set_block_dots(0)
    print("cuda-core", a["iterations"], a["values"], "tensor", b["iterations"], b["values"])
    assert len(a["values"]) > 0 and len(b["values"]) > 0
    # the same distinct values
    for u, v in ((a["values"], b["values"]), (b["values"], a["values"])):
        assert max(np.abs(v - x).min() for x in u) < 1e-9
    # Method 4 may keep one or two copies of an exactly degenerate value
    # depending on rounding: counts may differ only by such copies
    for r in (a, b):
        v = np.sort(r["values"])
        distinct = np.concatenate([[True], np.diff(v) > 1e-9])
        r["distinct"] = v[distinct]
    assert len(a["distinct"]) == len(b["distinct"])  # so any extra values are copies
    assert abs(a["iterations"] - b["iterations"]) <= skip
