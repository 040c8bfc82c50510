"""Python front end of libtbgpu.so, mirroring the reference's entry points.

The reference drives its eigensolver from C: ``setup_hamiltonian`` builds the
structure, the ``matmul`` function pointer (``matvect_mult``) applies H and
``eigensolve_lanczos`` runs the solver (nemo3d/src/base/eigsys3d_par.c:217-405,
eigen/src/lanczos.c:1823-2089).  ``Hamiltonian`` wraps one libtbgpu context
with the same three operations and the same argument meaning; failures raise
``TbgpuError`` carrying the library's status code.  There is no CPU path: if
the CUDA library or a GPU is missing, construction fails.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import materials as _mat

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtbgpu.so")

BAND_MODEL_IDS = {"sp3s*": 1, "sp3s*_so": 2, "sp3d5s*": 3, "sp3d5s*_so": 4}
NPAR = 68


class TbgpuError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = _lib().tbgpu_error_string(code).decode() if _LIB else str(code)
        super().__init__(f"{where}: {msg} (code {code})")


class _Geom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("periodic", C.c_int * 3), ("lattice", C.c_double * 3),
                ("type", C.c_void_p), ("dsp", C.c_void_p)]


class _Model(C.Structure):
    _fields_ = [("band_model", C.c_int), ("include_strain", C.c_int),
                ("passivate", C.c_int), ("dangling_shift", C.c_double),
                ("nspecies", C.c_int), ("par", C.c_void_p), ("par_ok", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("build_ms", C.c_double), ("solve_ms", C.c_double),
                ("vectors_ms", C.c_double), ("spmv_ms", C.c_double),
                ("spmv_launches", C.c_long), ("lanczos_iterations", C.c_long),
                ("kernel_launches", C.c_long), ("refine_ms", C.c_double),
                ("vec_segments", C.c_long), ("vec_mismatch", C.c_long),
                ("update_ms", C.c_double), ("check_ms", C.c_double), ("wait_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run nemo3d_b200.build.build() "
                               "(the CUDA library is required; there is no CPU path)")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.c_int, C.c_double
        L.tbgpu_error_string.restype = C.c_char_p
        L.tbgpu_error_string.argtypes = [ip]
        L.tbgpu_prepare_params.argtypes = [ip, ip, vp, vp, dp, dp, vp]
        L.tbgpu_set_bloch_k.argtypes = [vp, C.POINTER(C.c_double)]
        L.tbgpu_set_ham_precision.argtypes = [vp, ip]
        L.tbgpu_set_ham_storage.argtypes = [vp, ip]
        L.tbgpu_set_lanczos_precision.argtypes = [vp, ip]
        L.tbgpu_get_state_errors.argtypes = [vp, ip, vp, vp]
        L.tbgpu_hx_dev_f32.argtypes = [vp, dp, vp, vp]
        L.tbgpu_momentum_matrix.argtypes = [vp, ip, vp, vp, vp, vp]
        L.tbgpu_eigensolve_lanczos_batched.argtypes = [vp, ip, vp, ip, ip, ip, ip, ip, vp, vp,
                                                       vp, vp, dp, vp, vp, ip, vp, vp, vp, ip]
        L.tbgpu_vff_energy.argtypes = [vp, vp, vp, vp]
        L.tbgpu_vff_relax.argtypes = [vp, vp, ip, ip, dp, ip, vp, vp, vp]
        L.tbgpu_write_eigenvalues.argtypes = [C.c_char_p, C.c_char, vp, ip, vp]
        L.tbgpu_write_eigenvector.argtypes = [vp, C.c_char_p, vp, ip]
        L.tbgpu_hx_block_dev.argtypes = [vp, ip, dp, vp, vp]
        L.tbgpu_block_dots_dev.argtypes = [vp, ip, vp, vp, C.c_long, vp]
        L.tbgpu_set_block_dots.argtypes = [vp, ip]
        L.tbgpu_set_mixed_acceptance.argtypes = [vp, dp]
        L.tbgpu_release_solver_memory.argtypes = []
        L.tbgpu_eigensolve_blk_lanczos.argtypes = [vp, ip, ip, ip, ip, ip, dp, dp, dp, dp, dp,
                                                   ip, ip, vp, vp, vp, vp, vp, vp, ip]
        L.tbgpu_ctx_create.argtypes = [C.POINTER(_Geom), C.POINTER(_Model), C.POINTER(vp)]
        L.tbgpu_ctx_create_dev.argtypes = [C.POINTER(_Geom), C.POINTER(_Model), C.POINTER(vp)]
        L.tbgpu_ctx_destroy.argtypes = [vp]
        L.tbgpu_set_stream.argtypes = [vp, vp]
        L.tbgpu_build_hamiltonian.argtypes = [vp]
        L.tbgpu_num_atoms.restype = C.c_long
        L.tbgpu_num_atoms.argtypes = [vp]
        L.tbgpu_dimension.restype = C.c_long
        L.tbgpu_dimension.argtypes = [vp]
        L.tbgpu_matvect_mult.restype = None
        L.tbgpu_matvect_mult.argtypes = [C.POINTER(vp), vp, vp]
        L.tbgpu_hx_dev.argtypes = [vp, dp, vp, vp]
        L.tbgpu_eigensolve_lanczos.argtypes = [vp, ip, ip, ip, ip, ip, dp, dp, dp, dp, dp,
                                               vp, vp, vp, vp, vp, ip]
        L.tbgpu_eigensolve_lanczos_dev.argtypes = [vp, ip, ip, ip, ip, ip, dp, dp, dp, dp,
                                                   dp, vp, vp, vp, vp, vp, ip]
        L.tbgpu_get_tridiagonal.argtypes = [vp, vp, vp, ip]
        L.tbgpu_export_pattern.argtypes = [vp, vp, vp, vp]
        L.tbgpu_export_hamiltonian.argtypes = [vp, vp, vp]
        L.tbgpu_set_profiling.argtypes = [vp, ip]
        L.tbgpu_set_spmv_variant.argtypes = [vp, ip]
        L.tbgpu_autotune_spmv.argtypes = [vp, ip, vp, vp]
        L.tbgpu_set_start_vector.argtypes = [vp, vp]
        L.tbgpu_matvect_mult_dev.restype = None
        L.tbgpu_matvect_mult_dev.argtypes = [C.POINTER(vp), vp, vp]
        L.tbgpu_get_stats.argtypes = [vp, C.POINTER(Stats)]
        L.tbgpu_set_fold.argtypes = [vp, ip, dp, dp, dp, dp]
        L.tbgpu_matvect_mult2.restype = None
        L.tbgpu_matvect_mult2.argtypes = [C.POINTER(vp), vp, vp]
        L.tbgpu_hx_fold_dev.argtypes = [vp, vp, vp]
        L.tbgpu_get_fold_energies.argtypes = [vp, ip, vp]
        L.tbgpu_set_eigenvector_pass.argtypes = [vp, ip, ip, ip]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def release_solver_memory():
    """Return the device memory the solver's pools keep between solves
    (tbgpu_release_solver_memory); call once the solves have finished."""
    rc = _lib().tbgpu_release_solver_memory()
    if rc:
        raise TbgpuError(rc, "tbgpu_release_solver_memory")


def write_eigenvalues(path: str, mode: str, k, E):
    """nd_Ek file (tbgpu_write_eigenvalues): mode 'i' empties it, 'a' appends
    the eigenvalues E at Bloch vector k."""
    e = np.ascontiguousarray(np.asarray(E, np.float64))
    kv = np.ascontiguousarray(np.asarray(k if k is not None else (0, 0, 0), np.float64))
    rc = _lib().tbgpu_write_eigenvalues(path.encode(), mode.encode(), _p(kv), int(e.size),
                                        _p(e))
    if rc:
        raise TbgpuError(rc, "tbgpu_write_eigenvalues")


def prepare_params(mat: dict, include_strain: bool = True) -> np.ndarray:
    """param_init for one material set (nemo3d/src/base/mat3d.c:133-307)."""
    out = np.zeros(NPAR)
    pv = np.zeros(35)
    pv[:len(mat["pv"])] = mat["pv"]
    st = np.asarray(mat["strain"], np.float64)
    rc = _lib().tbgpu_prepare_params(int(mat["family"] == "sp3s*"), int(include_strain),
                                     _p(pv), _p(st), float(mat["ev_offset"]),
                                     float(mat["a0"]), _p(out))
    if rc:
        raise TbgpuError(rc, "prepare_params")
    return out


def param_table(mats, include_strain=True, nspecies=8):
    par = np.zeros((nspecies, nspecies, NPAR))
    ok = np.zeros((nspecies, nspecies), np.uint8)
    for m in mats:
        c, a = _mat.SPECIES[m["cation"]], _mat.SPECIES[m["anion"]]
        par[c, a] = prepare_params(m, include_strain)
        ok[c, a] = 1
    return par, ok


class Hamiltonian:
    """A structure's tight-binding Hamiltonian on the GPU (one libtbgpu context).

    ``structure``: a ``workloads.Structure``; ``model``: one of
    ``materials.BAND_MODELS``; ``materials``: parameter sets (default: every
    shipped set of the model's family).  ``ham_bits=32``: single-precision
    store; ``recompute=True``: blocks recomputed in every H*x;
    ``lanczos_bits=32`` (with ``ham_bits=32``): mixed-precision Lanczos with
    a double-precision refinement of the returned eigenpairs.
    """

    def __init__(self, structure, model="sp3d5s*_so", materials=None, include_strain=True,
                 passivate=True, dangling_shift=30.0, device_inputs=None, build=True,
                 ham_bits=64, recompute=False, lanczos_bits=64):
        L = _lib()
        self.structure = structure
        self.model = model
        self.norb, self.nspin = _mat.BAND_MODELS[model]
        self.nb = self.norb * self.nspin
        mats = materials if materials is not None else _mat.materials_for(model)
        if isinstance(mats, dict):
            mats = [mats]
        self._par, self._ok = param_table(mats, include_strain)
        g = _Geom()
        g.nx, g.ny, g.nz = structure.nx, structure.ny, structure.nz
        g.periodic[:] = [int(bool(v)) for v in structure.periodic]
        g.lattice[:] = list(structure.lattice)
        m = _Model()
        m.band_model = BAND_MODEL_IDS[model]
        m.include_strain, m.passivate = int(include_strain), int(passivate)
        m.dangling_shift = float(dangling_shift)
        m.nspecies = self._par.shape[0]
        m.par, m.par_ok = _p(self._par), _p(self._ok)
        ctx = C.c_void_p()
        if device_inputs is not None:  # (type_dev_ptr, dsp_dev_ptr or 0)
            g.type, g.dsp = device_inputs[0], (device_inputs[1] or None)
            rc = L.tbgpu_ctx_create_dev(C.byref(g), C.byref(m), C.byref(ctx))
        else:
            self._types = np.ascontiguousarray(structure.types, np.uint8)
            self._dsp = (None if structure.dsp is None
                         else np.ascontiguousarray(structure.dsp, np.float64))
            g.type, g.dsp = _p(self._types), _p(self._dsp)
            rc = L.tbgpu_ctx_create(C.byref(g), C.byref(m), C.byref(ctx))
        if rc:
            raise TbgpuError(rc, "tbgpu_ctx_create")
        self._ctx = ctx
        self._built = False
        # a failed option or build releases the context here, once (close()
        # clears the handle, so the destructor does not release it again)
        options = []
        if recompute:
            options.append(("tbgpu_set_ham_storage", 1))
        if ham_bits != 64:
            options.append(("tbgpu_set_ham_precision", int(ham_bits)))
        if lanczos_bits != 64:
            options.append(("tbgpu_set_lanczos_precision", int(lanczos_bits)))
        for name, value in options:
            rc = getattr(L, name)(ctx, value)
            if rc:
                self.close()
                raise TbgpuError(rc, name)
        if build:
            try:
                self.build()
            except TbgpuError:
                self.close()
                raise

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "_ctx", None):
            _lib().tbgpu_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        rc = _lib().tbgpu_set_stream(self._ctx, C.c_void_p(stream_ptr))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_stream")

    def build(self):
        rc = _lib().tbgpu_build_hamiltonian(self._ctx)
        if rc:
            raise TbgpuError(rc, "tbgpu_build_hamiltonian")
        self._built = True
        self.natoms = int(_lib().tbgpu_num_atoms(self._ctx))
        self.n = int(_lib().tbgpu_dimension(self._ctx))

    # -- H x ----------------------------------------------------------------
    def matvect_mult(self, x: np.ndarray, shift: float = 0.0) -> np.ndarray:
        """y = (H - shift) x through the reference's matmul signature."""
        x = np.ascontiguousarray(x, np.float64)
        if x.size != 2 * self.n:
            raise ValueError("x must hold 2*dimension doubles (interleaved complex)")
        y = np.empty_like(x)
        sh = C.c_double(shift)
        args = (C.c_void_p * 3)(self._ctx.value, C.cast(C.pointer(sh), C.c_void_p).value, None)
        L = _lib()
        L.tbgpu_matvect_mult(args, _p(y), _p(x))
        rc = L.tbgpu_last_error()
        if rc:
            raise TbgpuError(rc, "tbgpu_matvect_mult")
        return y

    def hx_dev(self, x_ptr: int, y_ptr: int, shift: float = 0.0):
        rc = _lib().tbgpu_hx_dev(self._ctx, float(shift), C.c_void_p(x_ptr), C.c_void_p(y_ptr))
        if rc:
            raise TbgpuError(rc, "tbgpu_hx_dev")

    def hx_dev_f32(self, x_ptr: int, y_ptr: int, shift: float = 0.0):
        """Mixed-precision product on complex-float device vectors."""
        rc = _lib().tbgpu_hx_dev_f32(self._ctx, float(shift), C.c_void_p(x_ptr),
                                     C.c_void_p(y_ptr))
        if rc:
            raise TbgpuError(rc, "tbgpu_hx_dev_f32")

    def hx_block_dev(self, p: int, x_ptr: int, y_ptr: int, shift: float = 0.0):
        """Y_v = (H - shift) X_v for p device vectors stored back to back."""
        rc = _lib().tbgpu_hx_block_dev(self._ctx, int(p), float(shift), C.c_void_p(x_ptr),
                                       C.c_void_p(y_ptr))
        if rc:
            raise TbgpuError(rc, "tbgpu_hx_block_dev")

    def block_dots_dev(self, p: int, x_ptr: int, y_ptr: int, n2: int):
        """G = X^H Y (p x p complex) of two blocks of p device vectors of n2
        complex entries stored back to back, on the tensor cores."""
        G = np.empty(2 * p * p)
        rc = _lib().tbgpu_block_dots_dev(self._ctx, int(p), C.c_void_p(x_ptr),
                                         C.c_void_p(y_ptr), int(n2), _p(G))
        if rc:
            raise TbgpuError(rc, "tbgpu_block_dots_dev")
        return (G[0::2] + 1j * G[1::2]).reshape(p, p)

    def set_mixed_acceptance(self, floor: float):
        """Mixed-precision solves: floor of the bound on the last components
        of a tridiagonal eigenvector that accepts its Ritz value (0: the
        solve's tolerance; negative: 2^-24 times the Gershgorin bound of the
        tridiagonal matrix, the complex-float rounding level)."""
        rc = _lib().tbgpu_set_mixed_acceptance(self._ctx, float(floor))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_mixed_acceptance")

    def set_block_dots(self, mode: int):
        """Block Lanczos dots on the CUDA cores in double (0) or on the tensor
        cores (1, int8 slices of the double entries)."""
        rc = _lib().tbgpu_set_block_dots(self._ctx, int(mode))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_block_dots")

    # -- eigensolver ----------------------------------------------------------
    def eigensolve_lanczos(self, r_0, ConvCheckStartIter=200, ConvCheckSkipRate=50,
                           imax=2400, requested1=1, requested2=1, emin1=-0.6, emax1=0.2,
                           emin2=1.4, emax2=2.0, tolerance=1e-7, vectors=0):
        """Lanczos with the reference's parameters (eigensolve_lanczos).

        r_0: host start vector (2*dimension doubles).  Returns a dict with
        ``values`` (ascending), ``conv_iterations``, ``iterations`` and, when
        ``vectors`` > 0, ``vectors`` (complex, [k, dimension])."""
        r0 = None if r_0 is None else np.ascontiguousarray(r_0, np.float64)
        if r0 is not None and r0.size != 2 * self.n:
            raise ValueError("r_0 must hold 2*dimension doubles")
        vals = np.zeros(imax)
        cit = np.zeros(imax, np.int32)
        its = np.zeros(1, np.int32)
        # the library writes interleaved (re, im) doubles: the layout of
        # complex128, so the result is a view of this array (no zero fill,
        # no second copy of what can be gigabytes)
        V = np.empty((vectors, 2 * self.n)) if vectors else None
        ne = _lib().tbgpu_eigensolve_lanczos(
            self._ctx, ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2,
            emin1, emax1, emin2, emax2, tolerance, _p(r0), _p(vals), _p(cit), _p(its),
            _p(V), int(vectors))
        if ne < 0:
            raise TbgpuError(ne, "tbgpu_eigensolve_lanczos")
        out = dict(values=vals[:ne].copy(), conv_iterations=cit[:ne].copy(),
                   iterations=int(its[0]))
        if vectors:
            k = min(ne, vectors)
            out["vectors"] = V[:k].view(np.complex128)
        return out

    def eigensolve_lanczos_batched(self, r_0, dot_cells, emin1, emax1, emin2, emax2,
                                   ConvCheckStartIter=200, ConvCheckSkipRate=50, imax=2400,
                                   requested1=1, requested2=1, tolerance=1e-7, vectors=0,
                                   values_stride=None):
        """Lanczos for the dots of a packed structure (``workloads.pack_dots``):
        ``dot_cells`` the cell boundaries along x, windows per dot (arrays, or
        scalars for all).  ``r_0``: host start vector (2*dimension doubles) or a
        CUDA tensor.  Returns a dict with ``values`` (list per dot, ascending),
        ``iterations`` per dot and, with ``vectors`` > 0, ``vectors``
        ([vectors, dimension] complex, the packed layout)."""
        import torch
        nd = len(dot_cells) - 1
        cells = np.ascontiguousarray(dot_cells, np.int32)
        win = [np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float64), (nd,)))
               for v in (emin1, emax1, emin2, emax2)]
        if isinstance(r_0, torch.Tensor) and r_0.is_cuda:
            r0 = r_0.contiguous()
        else:
            r0 = torch.from_numpy(np.ascontiguousarray(r_0, np.float64)).cuda()
        vs = values_stride or (requested1 + requested2 + 16)
        vals = np.zeros(nd * vs)
        found = np.zeros(nd, np.int32)
        its = np.zeros(nd, np.int32)
        V = torch.zeros(vectors * 2 * self.n, dtype=torch.float64, device="cuda") if vectors else None
        rc = _lib().tbgpu_eigensolve_lanczos_batched(
            self._ctx, nd, _p(cells), ConvCheckStartIter, ConvCheckSkipRate, imax, requested1,
            requested2, _p(win[0]), _p(win[1]), _p(win[2]), _p(win[3]), tolerance,
            C.c_void_p(r0.data_ptr()), _p(vals), vs, _p(found), _p(its),
            C.c_void_p(V.data_ptr()) if V is not None else None, int(vectors))
        if rc < 0:
            raise TbgpuError(rc, "tbgpu_eigensolve_lanczos_batched")
        out = dict(values=[vals[d * vs:d * vs + found[d]].copy() for d in range(nd)],
                   iterations=its.copy())
        if vectors:
            out["vectors"] = np.ascontiguousarray(V.cpu().numpy()).reshape(
                vectors, 2 * self.n).view(np.complex128)
        return out

    def eigensolve_lanczos_dev(self, r0_ptr: int, vectors_ptr: int = 0, max_vectors: int = 0,
                               ConvCheckStartIter=200, ConvCheckSkipRate=50, imax=2400,
                               requested1=1, requested2=1, emin1=-0.6, emax1=0.2, emin2=1.4,
                               emax2=2.0, tolerance=1e-7):
        vals = np.zeros(imax)
        cit = np.zeros(imax, np.int32)
        its = np.zeros(1, np.int32)
        ne = _lib().tbgpu_eigensolve_lanczos_dev(
            self._ctx, ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2,
            emin1, emax1, emin2, emax2, tolerance, C.c_void_p(r0_ptr), _p(vals), _p(cit),
            _p(its), C.c_void_p(vectors_ptr or None), int(max_vectors))
        if ne < 0:
            raise TbgpuError(ne, "tbgpu_eigensolve_lanczos_dev")
        return dict(values=vals[:ne].copy(), conv_iterations=cit[:ne].copy(),
                    iterations=int(its[0]))

    def tridiagonal(self, cap=100000):
        a = np.zeros(cap)
        b = np.zeros(cap)
        n = _lib().tbgpu_get_tridiagonal(self._ctx, _p(a), _p(b), cap)
        if n < 0:
            raise TbgpuError(n, "tbgpu_get_tridiagonal")
        return a[:n].copy(), b[:n].copy()

    # -- exports ----------------------------------------------------------------
    def export_pattern(self):
        site = np.zeros(self.natoms, np.int32)
        nbr = np.zeros(self.natoms * 4, np.int32)
        surf = np.zeros(self.natoms, np.uint8)
        rc = _lib().tbgpu_export_pattern(self._ctx, _p(site), _p(nbr), _p(surf))
        if rc:
            raise TbgpuError(rc, "tbgpu_export_pattern")
        return site, nbr, surf

    def export_hamiltonian(self):
        ons = np.zeros(self.natoms * self.nb * self.nb * 2)
        blk = np.zeros(self.natoms * 4 * self.norb * self.norb)
        rc = _lib().tbgpu_export_hamiltonian(self._ctx, _p(ons), _p(blk))
        if rc:
            raise TbgpuError(rc, "tbgpu_export_hamiltonian")
        return ons, blk

    def eigensolve_blk_lanczos(self, r0_block, ConvCheckStartIter=200, ConvCheckSkipRate=50,
                               imax=2000, requested1=1, requested2=1, emin1=-0.6, emax1=0.2,
                               emin2=1.4, emax2=2.0, tolerance=1e-7, max_no_success=0,
                               vectors=0):
        """Block Lanczos (eigensolve_blk_lanczos).  r0_block: host start block,
        shape (p, 2*dimension) doubles.  Returns values (ascending),
        found_vb, found_cb, iterations and, when ``vectors`` > 0, the
        eigenvectors (complex, [k, dimension])."""
        r0 = np.ascontiguousarray(r0_block, np.float64)
        p = r0.shape[0]
        if r0.ndim != 2 or r0.shape[1] != 2 * self.n:
            raise ValueError("r0_block must have shape (p, 2*dimension)")
        vals = np.zeros(max(1, requested1 + requested2))
        nv = min(vectors, requested1 + requested2)
        vec = np.zeros(2 * self.n * max(nv, 1)) if nv > 0 else None
        f1, f2, it = C.c_int(), C.c_int(), C.c_int()
        rc = _lib().tbgpu_eigensolve_blk_lanczos(
            self._ctx, ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2,
            emin1, emax1, emin2, emax2, tolerance, p, max_no_success, _p(r0), _p(vals),
            C.byref(f1), C.byref(f2), C.byref(it), _p(vec), nv)
        if rc < 0:
            raise TbgpuError(rc, "tbgpu_eigensolve_blk_lanczos")
        out = {"values": vals[:rc].copy(), "found_vb": f1.value, "found_cb": f2.value,
               "iterations": it.value}
        if nv > 0:
            k = min(rc, nv)
            out["vectors"] = vec[:2 * self.n * k].reshape(k, 2 * self.n).view(np.complex128)
        return out

    def write_eigenvector(self, path: str, vec, crystal_structure: int = 2):
        """Write one eigenvector (complex [dimension]) as the reference's
        nd_evec file (tbgpu_write_eigenvector)."""
        v = np.ascontiguousarray(np.asarray(vec, np.complex128))
        if v.size != self.n:
            raise ValueError("vector must hold dimension complex entries")
        rc = _lib().tbgpu_write_eigenvector(self._ctx, path.encode(), _p(v.view(np.float64)),
                                            int(crystal_structure))
        if rc:
            raise TbgpuError(rc, "tbgpu_write_eigenvector")

    def set_bloch_k(self, k):
        """Bloch vector (reference units) for periodic structures; None or
        zeros is the Gamma point (tbgpu_set_bloch_k)."""
        kv = None if k is None else (C.c_double * 3)(*[float(v) for v in k])
        rc = _lib().tbgpu_set_bloch_k(self._ctx, kv)
        if rc:
            raise TbgpuError(rc, "tbgpu_set_bloch_k")

    def set_spmv_variant(self, variant: int):
        """0: warp-staged cp.async kernel (default, 10 orbitals); 1: lane-gather; 2: 2-stage;
        3: two-cell units; 4: all cp.async; 5: lane per (atom, spin); 6: the same lanes
        on the pencil-interleaved layout; 7: 6 with block rows double-buffered in
        shared memory (32-bit store, spin-orbit, closed z, nz a multiple of 16); 8, 9: the
        lane-gather kernel of variant 1 with 4 and 2 warps per block (every model)."""
        rc = _lib().tbgpu_set_spmv_variant(self._ctx, int(variant))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_spmv_variant")

    def set_fold(self, on=True, shift1=1.38, shift2=1.58, factor=-10.0, offset=0.0):
        """Folded-spectrum operator F = factor (H - shift2)(H - shift1) + offset for
        the Lanczos solves (tbgpu_set_fold; the defaults are matvect_mult2's)."""
        rc = _lib().tbgpu_set_fold(self._ctx, int(bool(on)), C.c_double(shift1),
                                   C.c_double(shift2), C.c_double(factor), C.c_double(offset))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_fold")

    def matvect_mult2(self, x: np.ndarray) -> np.ndarray:
        """y = F x through the matvect_mult2 drop-in (host vectors)."""
        x = np.ascontiguousarray(x, np.float64)
        if x.size != 2 * self.n:
            raise ValueError("x must hold 2*dimension doubles")
        y = np.empty_like(x)
        args = (C.c_void_p * 3)(self._ctx.value, None, None)
        _lib().tbgpu_matvect_mult2(args, _p(y), _p(x))
        rc = _lib().tbgpu_last_error()
        if rc:
            raise TbgpuError(rc, "tbgpu_matvect_mult2")
        return y

    def fold_energies(self):
        """<v, H v> / <v, v> of the eigenvectors of the last folded solve."""
        out = np.zeros(4096)
        n = _lib().tbgpu_get_fold_energies(self._ctx, 4096, _p(out))
        if n < 0:
            raise TbgpuError(n, "tbgpu_get_fold_energies")
        return out[:n].copy()

    def set_eigenvector_pass(self, mode: int, columns: int = 4, segment: int = 256):
        """0: the reference's second run of the recurrence; 1: regenerate
        ``segment``-iteration segments from first-pass checkpoints,
        ``columns`` at a time (tbgpu_set_eigenvector_pass)."""
        rc = _lib().tbgpu_set_eigenvector_pass(self._ctx, int(mode), int(columns), int(segment))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_eigenvector_pass")

    def set_start_vector(self, r_0):
        """Keep a start vector in the context (tbgpu_set_start_vector); solves
        called with ``r_0=None`` use it.  None clears it."""
        if r_0 is None:
            rc = _lib().tbgpu_set_start_vector(self._ctx, None)
        else:
            self._start = np.ascontiguousarray(r_0, np.float64)
            if self._start.size != 2 * self.n:
                raise ValueError("r_0 must hold 2*dimension doubles")
            rc = _lib().tbgpu_set_start_vector(self._ctx, _p(self._start))
        if rc:
            raise TbgpuError(rc, "tbgpu_set_start_vector")

    def autotune_spmv(self, reps: int = 10):
        """Time every H*x variant on this structure and keep the fastest
        (tbgpu_autotune_spmv); returns (variant, ms per launch)."""
        v = C.c_int(-1)
        ms = C.c_double(0.0)
        rc = _lib().tbgpu_autotune_spmv(self._ctx, int(reps), C.byref(v), C.byref(ms))
        if rc:
            raise TbgpuError(rc, "tbgpu_autotune_spmv")
        return v.value, ms.value

    def set_profiling(self, on=True):
        _lib().tbgpu_set_profiling(self._ctx, int(bool(on)))

    # -- Keating strain (before build) ---------------------------------------
    def vff_energy(self, vff=None, grad=False):
        """Keating energy at the current displacements and, with ``grad``,
        the reference's gradient per site ([nx, ny, nz, 8, 3])."""
        t = np.ascontiguousarray(_mat.vff_table() if vff is None else vff, np.float64)
        e = np.zeros(1)
        g = np.zeros(self.structure.nsites * 3) if grad else None
        rc = _lib().tbgpu_vff_energy(self._ctx, _p(t), _p(e), _p(g))
        if rc:
            raise TbgpuError(rc, "tbgpu_vff_energy")
        if grad:
            st = self.structure
            return float(e[0]), g.reshape(st.nx, st.ny, st.nz, 8, 3)
        return float(e[0])

    def vff_relax(self, vff=None, bc=0, max_iter=10000, tol=1e-9, end_if_small_step=1):
        """Relax the displacements with the Keating model (macopt); returns
        (displacements [nx, ny, nz, 8, 3], energy, iterations).  The build
        that follows uses the relaxed displacements."""
        t = np.ascontiguousarray(_mat.vff_table() if vff is None else vff, np.float64)
        st = self.structure
        d = np.zeros(st.nsites * 3)
        e = np.zeros(1)
        its = np.zeros(1, np.int32)
        rc = _lib().tbgpu_vff_relax(self._ctx, _p(t), int(bc), int(max_iter), float(tol),
                                    int(end_if_small_step), _p(e), _p(its), _p(d))
        if rc:
            raise TbgpuError(rc, "tbgpu_vff_relax")
        return d.reshape(st.nx, st.ny, st.nz, 8, 3), float(e[0]), int(its[0])

    def momentum_matrix(self, psi, E=None):
        """Optical momentum matrix elements of the states ``psi`` (complex
        [n, dimension], host or a CUDA tensor of 2*n*dimension doubles):
        returns P [3, n, 8n] complex in the reference's pXmatrix layout and,
        with eigenvalues ``E``, the transition table [3, n(n-1)/2, 4]."""
        import torch
        if isinstance(psi, torch.Tensor) and psi.is_cuda:
            dev = psi.contiguous()
            n = dev.numel() // (2 * self.n)
        else:
            a = np.asarray(psi, complex).reshape(-1, self.n)
            n = a.shape[0]
            dev = torch.from_numpy(np.stack([a.real, a.imag], -1).reshape(-1).copy()).cuda()
        P = np.zeros((3, n, 8 * n, 2))
        T = np.zeros((3, max(n * (n - 1) // 2, 1), 4)) if E is not None else None
        e = np.ascontiguousarray(E, np.float64) if E is not None else None
        rc = _lib().tbgpu_momentum_matrix(self._ctx, n, C.c_void_p(dev.data_ptr()), _p(e),
                                          _p(P), _p(T))
        if rc:
            raise TbgpuError(rc, "tbgpu_momentum_matrix")
        P = P[..., 0] + 1j * P[..., 1]
        return (P, T[:, :n * (n - 1) // 2] if T is not None else None)

    def state_errors(self):
        """Mixed-precision solve: per state with an eigenvector, the residual
        ||H v - lambda v|| of the refined pair and the change of the eigenvalue
        made by the double-precision refinement."""
        cap = 4096
        r, d = np.zeros(cap), np.zeros(cap)
        n = _lib().tbgpu_get_state_errors(self._ctx, cap, _p(r), _p(d))
        if n < 0:
            raise TbgpuError(n, "tbgpu_get_state_errors")
        return r[:n].copy(), d[:n].copy()

    def stats(self) -> dict:
        s = Stats()
        rc = _lib().tbgpu_get_stats(self._ctx, C.byref(s))
        if rc:
            raise TbgpuError(rc, "tbgpu_get_stats")
        return s.as_dict()
