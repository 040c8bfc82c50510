"""The eigensolve_lanczos drop-in (reference signature) on the GPU.

Calls ``eigensolve_lanczos`` of tests/shim/_build/libtbgpu_shim.so (the
drop-in of nemo3d_b200/shim/eigensolve_lanczos_tbgpu.c, built against the
reference's declaration) through its reference signature, with the libtbgpu
context in argument[0].

Bars:
* the returned count, *pValue (ascending) and the iteration count equal
  tbgpu_eigensolve_lanczos's on the same inputs, bit for bit;
* the saved state files have the reference's layout: the tridiagonal file's
  iterations, processors and alpha/beta interleaving equal the solve's
  tridiagonal matrix; the eigenvalue file holds the values;
* the eigenvectors in *pCVector agree with tbgpu_eigensolve_lanczos's
  (|<a, b>| within 1e-8 of 1) and *pCValue holds (value, 0);
* restoreState = 1 reads the files back (the reference's iterations - 200),
  returns the saved eigenvalues exactly, and its eigenvectors have residuals
  ||H v - lambda v|| below 1e-4 eV through the oracle's product.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "shim", "_build", "libtbgpu_shim.so")
MATS = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]


class DComplex(C.Structure):
    _fields_ = [("r", C.c_double), ("i", C.c_double)]


def _shim():
    if not os.path.exists(SHIM):
        pytest.fail("tests/shim/_build/libtbgpu_shim.so missing: run tests/shim/build_shim.sh")
    lib = C.CDLL(SHIM)
    f = lib.eigensolve_lanczos
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.POINTER(C.c_double)), C.c_int, C.c_int, C.c_int, C.c_int,
                  C.c_int, C.c_size_t, C.POINTER(C.c_void_p), C.c_double, C.c_double,
                  C.c_double, C.c_double, C.c_double, C.c_int, C.c_char_p, C.c_char_p,
                  C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.POINTER(DComplex)), C.POINTER(C.POINTER(C.POINTER(DComplex))),
                  C.c_void_p, C.c_int]
    return f


KW = dict(ConvCheckStartIter=100, ConvCheckSkipRate=50, imax=3000, requested1=2,
          requested2=3, emin1=-0.6, emax1=0.75, emin2=1.5, emax2=2.6, tolerance=1e-7)


def _call(f, g, r0, tmp, restore):
    n = g.n
    start = np.ascontiguousarray(r0, np.float64)
    r_n, q_n, q_n1 = start.copy(), np.zeros_like(start), np.zeros_like(start)
    args = (C.c_void_p * 3)(g._ctx.value, None, None)
    pv = C.POINTER(C.c_double)()
    pcv = C.POINTER(DComplex)()
    pvec = C.POINTER(C.POINTER(DComplex))()
    ne = f(C.byref(pv), KW["ConvCheckStartIter"], KW["ConvCheckSkipRate"], KW["imax"],
           KW["requested1"], KW["requested2"], n, args, KW["emin1"], KW["emax1"],
           KW["emin2"], KW["emax2"], KW["tolerance"], 0, None,
           os.path.join(tmp, "tridiag.bin").encode(), os.path.join(tmp, "eigval.bin").encode(),
           r_n.ctypes.data, start.ctypes.data, q_n.ctypes.data, q_n1.ctypes.data,
           C.byref(pcv), C.byref(pvec), None, int(restore))
    assert ne > 0, ne
    vals = np.array([pv[k] for k in range(ne)])
    cvals = np.array([[pcv[k].r, pcv[k].i] for k in range(ne)])
    vecs = []
    for k in range(ne):
        row = np.ctypeslib.as_array(C.cast(pvec[k], C.POINTER(C.c_double)), shape=(2 * n,))
        vecs.append(row[0::2] + 1j * row[1::2])
    return ne, vals, cvals, np.array(vecs)


def test_shim_solve_save_and_restore(tmp_path):
    from nemo3d_b200.tbgpu import Hamiltonian
    f = _shim()
    st = workloads.dome_in_box(cells=(8, 8, 6), base_nm=3.0, height_nm=1.2, wl_z_nm=1.2,
                               sigma_frac=0.01, seed=2)
    g = Hamiltonian(st, "sp3d5s*_so", MATS)
    r0 = workloads.random_start(g.n, seed=0)
    ref = g.eigensolve_lanczos(r0, vectors=8, **KW)
    tmp = str(tmp_path)
    ne, vals, cvals, vecs = _call(f, g, r0, tmp, restore=False)
    assert ne == len(ref["values"])
    np.testing.assert_array_equal(vals, ref["values"])
    np.testing.assert_array_equal(cvals[:, 0], vals)
    assert np.all(cvals[:, 1] == 0.0)
    for a, b in zip(vecs, ref["vectors"]):
        ov = abs(np.vdot(a, b)) / (np.linalg.norm(a) * np.linalg.norm(b))
        assert abs(ov - 1.0) < 1e-8, ov
    # the saved state, in the reference's layout
    raw = open(os.path.join(tmp, "tridiag.bin"), "rb").read()
    its, procs = np.frombuffer(raw[:8], np.int32)
    t = np.frombuffer(raw[8:], np.float64)
    a, b = g.tridiagonal()
    assert its == ref["iterations"] == len(a) and procs == 1 and t.size == 2 * its
    np.testing.assert_array_equal(t[0::2], a)
    np.testing.assert_array_equal(t[1:-1:2], b[:its - 1])
    ev = open(os.path.join(tmp, "eigval.bin"), "rb").read()
    assert np.frombuffer(ev[:4], np.int32)[0] == ne
    np.testing.assert_array_equal(np.frombuffer(ev[4:], np.float64), vals)
    # restoreState: the saved eigenvalues, eigenvectors from the stored
    # matrix less its last 200 iterations
    ne2, vals2, _, vecs2 = _call(f, g, r0, tmp, restore=True)
    assert ne2 == ne
    np.testing.assert_array_equal(vals2, vals)
    o = oracle.OracleHamiltonian(st, 10, 2, MATS)
    checked = 0
    for lam, v, cit in zip(vals2, vecs2, ref["conv_iterations"]):
        if cit > its - 200:  # converged within the iterations the restore drops
            continue
        checked += 1
        x = np.empty(2 * g.n)
        x[0::2], x[1::2] = v.real, v.imag
        hv = o.hx(x)
        r = np.linalg.norm((hv[0::2] + 1j * hv[1::2]) - lam * v) / np.linalg.norm(v)
        print("restored eigenpair", lam, "residual", r)
        assert r < 1e-4, (lam, r)
    assert checked >= 2
