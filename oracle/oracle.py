"""ctypes front end of the CPU oracle (oracle/tb_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke`` as
the checker and by the CPU-baseline leg of ``bench.py``.  The product never
imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
NPV, NSTR = 35, 33
NPAR = NPV + NSTR


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "tb_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", LIB,
                               src, "-lm"], cwd=HERE)
    return LIB


class _Geom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("periodic", C.c_int * 3), ("lattice", C.c_double * 3),
                ("type", C.c_void_p), ("dsp", C.c_void_p)]


class _Model(C.Structure):
    _fields_ = [("norb", C.c_int), ("nspin", C.c_int), ("include_strain", C.c_int),
                ("passivate", C.c_int), ("dangling_shift", C.c_double),
                ("nspecies", C.c_int), ("par", C.c_void_p), ("par_ok", C.c_void_p)]


class _Opts(C.Structure):
    _fields_ = [("conv_start", C.c_int), ("conv_skip", C.c_int), ("imax", C.c_int),
                ("req1", C.c_int), ("req2", C.c_int),
                ("emin1", C.c_double), ("emax1", C.c_double),
                ("emin2", C.c_double), ("emax2", C.c_double),
                ("tolerance", C.c_double), ("seed", C.c_uint)]


class _Ham(C.Structure):
    _fields_ = [("norb", C.c_int), ("nspin", C.c_int), ("natoms", C.c_long),
                ("atom_slot", C.c_void_p), ("nbr", C.c_void_p), ("wrap", C.c_void_p),
                ("kvec", C.c_void_p), ("onsite", C.c_void_p), ("blocks", C.c_void_p),
                ("shift", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        L.orc_prepare_params.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_double, C.c_double, C.c_void_p]
        L.orc_topology.restype = C.c_long
        L.orc_topology.argtypes = [C.POINTER(_Geom), C.c_long, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
        L.orc_build.argtypes = [C.POINTER(_Geom), C.POINTER(_Model), C.c_long,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_hx.argtypes = [C.c_int, C.c_int, C.c_long] + [C.c_void_p] * 6 + \
            [C.c_double, C.c_void_p, C.c_void_p]
        L.orc_dense.argtypes = [C.c_int, C.c_int, C.c_long] + [C.c_void_p] * 7
        L.orc_tridiag_eigs.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                       C.c_double, C.c_double, C.c_void_p]
        L.orc_eigensolve_lanczos.argtypes = [C.c_void_p, C.c_void_p, C.c_long,
                                             C.c_void_p, C.POINTER(_Opts), C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p]
        L.orc_onsite_block.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_bond.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_vff_energy.restype = C.c_double
        L.orc_vff_energy.argtypes = [C.POINTER(_Geom), C.c_long, C.c_void_p, C.c_void_p,
                                     C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_vff_free_mask.argtypes = [C.POINTER(_Geom), C.c_long, C.c_void_p, C.c_void_p,
                                        C.c_int, C.c_void_p]
        L.orc_vff_relax.argtypes = [C.POINTER(_Geom), C.c_long, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                    C.c_double, C.c_int, C.c_void_p, C.c_void_p]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def prepare_params(mat: dict, include_strain: bool = True) -> np.ndarray:
    out = np.zeros(NPAR)
    pv = np.zeros(NPV)
    pv[:len(mat["pv"])] = mat["pv"]
    st = np.asarray(mat["strain"], dtype=np.float64)
    lib().orc_prepare_params(int(mat["family"] == "sp3s*"), int(include_strain),
                             _p(pv), _p(st), float(mat["ev_offset"]),
                             float(mat["a0"]), _p(out))
    return out


def param_table(materials, include_strain=True, nspecies=8):
    """[ns, ns, NPAR] table indexed (cation species, anion species)."""
    from nemo3d_b200.materials import SPECIES
    par = np.zeros((nspecies, nspecies, NPAR))
    ok = np.zeros((nspecies, nspecies), dtype=np.uint8)
    for m in materials:
        c, a = SPECIES[m["cation"]], SPECIES[m["anion"]]
        par[c, a] = prepare_params(m, include_strain)
        ok[c, a] = 1
    return par, ok


class OracleHamiltonian:
    """Topology + assembled stored Hamiltonian of a structure."""

    def __init__(self, st, norb, nspin, materials, include_strain=True,
                 passivate=True, dangling_shift=30.0, kvec=None):
        self.st, self.norb, self.nspin = st, norb, nspin
        self.nb = norb * nspin
        self.types = np.ascontiguousarray(st.types, dtype=np.uint8).reshape(-1)
        self.dsp = None if st.dsp is None else np.ascontiguousarray(st.dsp, np.float64).reshape(-1)
        g = _Geom()
        g.nx, g.ny, g.nz = st.nx, st.ny, st.nz
        g.periodic[:] = [int(bool(x)) for x in st.periodic]
        g.lattice[:] = list(st.lattice)
        g.type = _p(self.types)
        g.dsp = _p(self.dsp)
        self._g = g
        ns = st.nsites
        slot = np.zeros(ns, np.int32)
        nbr = np.zeros(ns * 4, np.int32)
        wrap = np.zeros(ns * 12, np.int8)
        surf = np.zeros(ns, np.uint8)
        na = lib().orc_topology(C.byref(g), ns, _p(slot), _p(nbr), _p(wrap), _p(surf))
        self.natoms = int(na)
        self.atom_slot = slot[:na].copy()
        self.nbr = nbr[:na * 4].copy()
        self.wrap = wrap[:na * 12].copy()
        self.surface = surf[:na].copy()
        self.par, self.par_ok = param_table(materials, include_strain)
        m = _Model()
        m.norb, m.nspin, m.include_strain = norb, nspin, int(include_strain)
        m.passivate, m.dangling_shift = int(passivate), float(dangling_shift)
        m.nspecies = self.par.shape[0]
        m.par, m.par_ok = _p(self.par), _p(self.par_ok)
        self._m = m
        self.onsite = np.zeros(self.natoms * self.nb * self.nb * 2)
        self.blocks = np.zeros(self.natoms * 4 * norb * norb)
        rc = lib().orc_build(C.byref(g), C.byref(m), self.natoms, _p(self.atom_slot),
                             _p(self.nbr), _p(self.wrap), _p(self.surface),
                             _p(self.onsite), _p(self.blocks))
        if rc != 0:
            raise ValueError(f"orc_build failed ({rc}): missing material set")
        self.kvec = None if kvec is None else np.asarray(kvec, np.float64)
        self.n = self.natoms * self.nb

    def hx(self, x, shift=0.0):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        lib().orc_hx(self.norb, self.nspin, self.natoms, _p(self.atom_slot), _p(self.nbr),
                     _p(self.wrap), _p(self.kvec), _p(self.onsite), _p(self.blocks),
                     float(shift), _p(x), _p(y))
        return y

    def dense(self, kvec=None):
        k = None if kvec is None else np.asarray(kvec, np.float64)
        h = np.zeros(self.n * self.n * 2)
        lib().orc_dense(self.norb, self.nspin, self.natoms, _p(self.atom_slot), _p(self.nbr),
                        _p(self.wrap), _p(k), _p(self.onsite), _p(self.blocks), _p(h))
        h = h.reshape(self.n, self.n, 2)
        return h[..., 0] + 1j * h[..., 1]

    def lanczos(self, r0, imax=2000, req=(1, 1), erange1=(-1, 0), erange2=(1, 2),
                tol=1e-7, conv_start=200, conv_skip=50, eigvecs=False, seed=1,
                shift=0.0):
        """eigensolve_lanczos with this Hamiltonian; returns a dict."""
        ham = _Ham()
        ham.norb, ham.nspin, ham.natoms = self.norb, self.nspin, self.natoms
        ham.atom_slot, ham.nbr, ham.wrap = _p(self.atom_slot), _p(self.nbr), _p(self.wrap)
        ham.kvec, ham.onsite, ham.blocks = _p(self.kvec), _p(self.onsite), _p(self.blocks)
        ham.shift = float(shift)
        o = _Opts(conv_start, conv_skip, imax, req[0], req[1], erange1[0], erange1[1],
                  erange2[0], erange2[1], tol, seed)
        r0 = np.ascontiguousarray(r0, np.float64)
        ev = np.zeros(imax)
        cit = np.zeros(imax, np.int32)
        its = np.zeros(1, np.int32)
        al = np.zeros(imax)
        be = np.zeros(imax)
        nev_max = imax
        vec = np.zeros(2 * self.n * min(nev_max, 64)) if eigvecs else None
        fn = C.cast(lib().orc_ham_matvec, C.c_void_p)
        ne = lib().orc_eigensolve_lanczos(fn, C.byref(ham), self.n, _p(r0), C.byref(o),
                                          _p(ev), _p(cit), _p(its), _p(vec), _p(al), _p(be))
        it = int(its[0])
        out = dict(evals=ev[:ne].copy(), conv_it=cit[:ne].copy(), iterations=it,
                   alpha=al[:it].copy(), beta=be[:it].copy())
        if eigvecs:
            v = vec[:2 * self.n * ne].reshape(ne, self.n, 2)
            out["evecs"] = v[..., 0] + 1j * v[..., 1]
        return out


class _OracleH(C.Structure):
    _fields_ = [("norb", C.c_int), ("nspin", C.c_int), ("natoms", C.c_long),
                ("atom_slot", C.c_void_p), ("nbr", C.c_void_p), ("wrap", C.c_void_p),
                ("kvec", C.c_void_p), ("onsite", C.c_void_p), ("blocks", C.c_void_p)]


_REF_LANCZOS = None
REF_LANCZOS_PATH = os.path.join(HERE, "_ref", "libref_lanczos.so")


def ref_lanczos_available() -> bool:
    return os.path.exists(REF_LANCZOS_PATH)


def ref_eigenvalues_lanczos(o, r0, imax=2000, req=(1, 1), erange1=(-1, 0), erange2=(1, 2),
                            tol=1e-7, conv_start=200, conv_skip=50):
    """The reference's own first Lanczos pass (eigenvaluesLanczos of
    eigen/src/lanczos.c, compiled from its source into
    oracle/_ref/libref_lanczos.so by oracle/build_ref.sh) on the oracle's
    stored Hamiltonian ``o`` (its H*x as the reference's matmul).  Returns
    dict(evals, conv_it, iterations)."""
    global _REF_LANCZOS
    if _REF_LANCZOS is None:
        L = C.CDLL(REF_LANCZOS_PATH)
        L.ref_eigenvalues_lanczos.restype = C.c_int
        L.ref_eigenvalues_lanczos.argtypes = [
            C.c_void_p, C.c_long, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
            C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
            C.c_void_p]
        _REF_LANCZOS = L
    h = _OracleH(o.norb, o.nspin, o.natoms, _p(o.atom_slot), _p(o.nbr), _p(o.wrap),
                 _p(o.kvec), _p(o.onsite), _p(o.blocks))
    r0 = np.ascontiguousarray(r0, np.float64)
    ev = np.zeros(imax)
    cit = np.zeros(imax, np.int32)
    its = np.zeros(1, np.int32)
    ne = _REF_LANCZOS.ref_eigenvalues_lanczos(
        C.byref(h), o.n, _p(r0), conv_start, conv_skip, imax, req[0], req[1], erange1[0],
        erange1[1], erange2[0], erange2[1], tol, _p(ev), _p(cit), _p(its))
    return dict(evals=ev[:ne].copy(), conv_it=cit[:ne].copy(), iterations=int(its[0]))


_REF_BLK = None


def ref_block_lanczos(o, r0_block, imax=400, req=(0, 1), erange1=(-1, 0), erange2=(1, 2),
                      tol=1e-7, conv_start=200, conv_skip=50, max_no_success=0):
    """The reference's own block Lanczos eigenvalue pass (block_Lanczos_QR
    and block_lanczos_blocktridiagonal of eigen/src/lanczos_blk.c, compiled
    from its source into oracle/_ref/libref_lanczos.so by
    oracle/build_ref.sh) from the start block r0_block (p rows of 2n doubles)
    on the oracle's stored Hamiltonian ``o``.  Returns dict(evals, found_vb,
    found_cb, iterations).  The routine prints progress on stdout.

    Its valence window (window 1) reports W[M-i], i = 0.., of zhbevx's M
    values (lanczos_blk.c:960-975): one entry past the values found, which
    zhbevx leaves unset, comes first and the highest value is dropped.  Pins
    therefore use window 2 (W[i], the lowest values of its range), placed
    over whichever energies they test."""
    global _REF_BLK
    if _REF_BLK is None:
        L = C.CDLL(REF_LANCZOS_PATH)
        L.ref_block_lanczos.restype = C.c_int
        L.ref_block_lanczos.argtypes = [
            C.c_void_p, C.c_long, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
            C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _REF_BLK = L
    h = _OracleH(o.norb, o.nspin, o.natoms, _p(o.atom_slot), _p(o.nbr), _p(o.wrap),
                 _p(o.kvec), _p(o.onsite), _p(o.blocks))
    r0 = np.ascontiguousarray(r0_block, np.float64)
    p = r0.shape[0]
    ev = np.zeros(imax * p)
    fvb = np.zeros(1, np.int32)
    fcb = np.zeros(1, np.int32)
    its = np.zeros(1, np.int32)
    ne = _REF_BLK.ref_block_lanczos(
        C.byref(h), o.n, p, _p(r0), conv_start, conv_skip, imax, req[0], req[1], erange1[0],
        erange1[1], erange2[0], erange2[1], tol, max_no_success, _p(ev), _p(fvb), _p(fcb),
        _p(its))
    return dict(evals=ev[:ne].copy(), found_vb=int(fvb[0]), found_cb=int(fcb[0]),
                iterations=int(its[0]))


def tridiag_eigs(d, e, vl, vu, abstol=1e-13):
    d = np.ascontiguousarray(d, np.float64)
    e = np.ascontiguousarray(e, np.float64)
    w = np.zeros(len(d))
    n = lib().orc_tridiag_eigs(len(d), _p(d), _p(e), vl, vu, abstol, _p(w))
    return w[:n].copy()


def block_lanczos(hx, r0_block, imax=400, req=(1, 1), erange1=(-1, 0), erange2=(1, 2),
                  tol=1e-7, conv_start=200, conv_skip=50, max_no_success=0):
    """eigensolve_blk_lanczos restated with numpy (test infrastructure only).

    Follows NEMO_3D/eigen/src/lanczos_blk.c: block_Lanczos_QR (273-357,
    modified Gram-Schmidt), single_iteration (392-550, no deflation),
    block_lanczos_blocktridiagonal (1412-1678: band storage, checks every
    conv_skip steps after conv_start, n_nosuccess, stop rule) and
    find_block_converged_eigvalues_Method4 (553-634).  The window
    eigenvalues of the band matrix come from numpy's dense Hermitian solver
    (the reference calls zhbevx).  In the valence window the reference takes
    W[M-i], i = 0.., one past the last value found; this takes the highest
    values W[M-1-i].  hx(x) maps a complex vector to H x.
    """
    Rb = np.array([r[0::2] + 1j * r[1::2] for r in np.asarray(r0_block, np.float64)])
    p, n = Rb.shape

    def qr(R):
        Q = np.zeros_like(R)
        B = np.zeros((p, p), complex)
        g = np.sqrt(np.vdot(R[0], R[0]).real)
        B[0, 0] = g
        Q[0] = R[0] / g
        for i in range(1, p):
            r2 = R[i].copy()
            for k in range(i):
                b = np.vdot(Q[k], r2)
                B[k, i] = b
                r2 = r2 - b * Q[k]
            g = np.sqrt(np.vdot(r2, r2).real)
            B[i, i] = g
            Q[i] = r2 / g
        return Q, B

    Q, _ = qr(Rb)
    Qo = np.zeros_like(Q)
    blocks_a, blocks_b = [], []
    old1, old2, conv1, conv2 = [], [], [], []
    nos = [0, 0]
    mns = max_no_success if max_no_success > 0 else 1 << 30
    skip, it = 0, 0

    def method4(fresh, old, conv, requested, k):
        tmp, olds = [], list(old)
        for v in fresh:
            for jj, o in enumerate(olds):
                if abs(v - o) < tol:
                    tmp.append(v)
                    olds[jj] = 500.0
                    break
            if len(tmp) == requested:
                break
        for ci in range(len(conv)):
            for tj in range(len(tmp)):
                if abs(conv[ci] - tmp[tj]) < 100 * tol:
                    conv[ci] = tmp[tj]
                    tmp[tj] = 500.0
                    break
        for t in tmp:
            if abs(t) < 490.0:
                conv.append(t)
                nos[k] = 0
                if len(conv) == requested:
                    break
        old[:] = fresh

    def window(T, lo, hi):
        w = np.linalg.eigvalsh(T)
        return w[(w > lo) & (w <= hi)]

    B = None
    while True:
        if it != 0:
            Q, B = qr(Rb)
        Rb = np.array([hx(q) for q in Q])
        if it != 0:
            Rb = Rb - (B.conj() @ Qo)           # R_i -= sum_k conj(B[i,k]) Qold_k
        A = np.array([[np.vdot(Q[i], Rb[j]) for j in range(p)] for i in range(p)])
        A = np.tril(A) + np.tril(A, -1).conj().T
        A[np.diag_indices(p)] = A.diagonal().real
        Rb = Rb - A.T @ Q                        # R_i -= sum_k Q_k A[k, i]
        Qo = Q
        blocks_a.append(A)
        if it != 0:
            blocks_b.append(B)
        skip += 1
        if conv_start < it:
            if len(conv1) < req[0]:
                nos[0] += 1
            if len(conv2) < req[1]:
                nos[1] += 1
        if conv_start < it and conv_skip <= skip:
            skip = 0
            m = len(blocks_a)
            T = np.zeros((m * p, m * p), complex)
            for k, Ak in enumerate(blocks_a):
                T[k * p:(k + 1) * p, k * p:(k + 1) * p] = Ak
            for k, Bk in enumerate(blocks_b):   # coupling of block k+1 to block k
                T[(k + 1) * p:(k + 2) * p, k * p:(k + 1) * p] = np.triu(Bk)
                T[k * p:(k + 1) * p, (k + 1) * p:(k + 2) * p] = np.triu(Bk).conj().T
            if req[0] > 0 and len(conv1) < req[0]:
                w = window(T, *erange1)
                method4(list(w[::-1][:req[0] + 1]), old1, conv1, req[0], 0)
            if req[1] > 0 and len(conv2) < req[1]:
                w = window(T, *erange2)
                method4(list(w[:req[1] + 1]), old2, conv2, req[1], 1)
        done = (len(conv1) >= req[0] and len(conv2) >= req[1]) or it + 2 == imax
        stalled = nos[0] >= mns or nos[1] >= mns
        it += 1
        if done or stalled or it + 1 >= imax:
            break
    return dict(evals=np.sort(np.array(conv1 + conv2)), found_vb=len(conv1),
                found_cb=len(conv2), iterations=it)


def kramers_partner(v, norb):
    """Time-reversal partner of a spin state as eigsys3d_par.c:461-475 writes
    it: up <- -conj(down), down <- conj(up), per atom."""
    v = np.asarray(v, complex).reshape(-1, 2 * norb)
    w = np.empty_like(v)
    w[:, norb:] = np.conj(v[:, :norb])
    w[:, :norb] = -np.conj(v[:, norb:])
    return w.reshape(-1)


def momentum_matrix(o, psi, E=None):
    """Momentum (optical) matrix elements, literally as the reference's
    MOMENTUM_MATRIX block computes them (eigsys3d_par.c:410-640, the same code
    for Px, Py, Pz): for final state f, H psi_f, H psi'_f, x H psi, x H psi',
    x psi, x psi', H x psi, H x psi' (psi' the Kramers partner, x the strained
    atom coordinate); for initial state i, temp1 = <a|x H b>, temp2 = <a|H x b>
    and p = i (temp2 - temp1) for (a, b) in (psi_i, psi_f), (psi_i, psi'_f),
    (psi'_i, psi_f), (psi'_i, psi'_f).  Returns P [3][n][8n] complex in the
    pXmatrix layout (labels (+-(i+1), +-(f+1)) before each value) and, when E
    is given, the transition table [3][n(n-1)/2][4] (istate, fstate,
    E_i - E_f, sum of |p|^2 over the four pairs) for istate > fstate in the
    order the reference fills TransProbX (fstate outer)."""
    psi = [np.asarray(p, complex).reshape(-1) for p in psi]
    n, nb, norb = len(psi), o.nb, o.norb
    pos = o.st.site_positions().reshape(-1, 3)[o.atom_slot]
    if o.st.dsp is not None:
        pos = pos + np.asarray(o.st.dsp, np.float64).reshape(-1, 3)[o.atom_slot]

    def H(v):
        x = np.stack([v.real, v.imag], -1).reshape(-1)
        y = o.hx(x).reshape(-1, 2)
        return y[:, 0] + 1j * y[:, 1]

    P = np.zeros((3, n, 8 * n), complex)
    T = np.zeros((3, n * (n - 1) // 2, 4)) if E is not None else None
    for d in range(3):
        r = np.repeat(pos[:, d], nb)
        k = 0
        for f in range(n):
            bf = [psi[f], kramers_partner(psi[f], norb)]
            Hb = [H(b) for b in bf]
            xHb = [r * h for h in Hb]
            Hxb = [H(r * b) for b in bf]
            for i in range(n):
                ai = [psi[i], kramers_partner(psi[i], norb)]
                for c, (ia, fb) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
                    t1 = np.vdot(ai[ia], xHb[fb])
                    t2 = np.vdot(ai[ia], Hxb[fb])
                    P[d, i, 8 * f + 2 * c] = complex((i + 1) * (-1 if ia else 1),
                                                     (f + 1) * (-1 if fb else 1))
                    P[d, i, 8 * f + 2 * c + 1] = complex(t1.imag - t2.imag, t2.real - t1.real)
                if T is not None and i > f:
                    vals = P[d, i, 8 * f + 1:8 * f + 8:2]
                    T[d, k] = (i + 1, f + 1, E[i] - E[f], float(np.sum(np.abs(vals) ** 2)))
                    k += 1
    return P, T


class OracleVFF:
    """Keating valence-force-field strain of a structure (the reference's
    min_estrain with StrainModel = VFF_keating; see tb_oracle.h).
    ``vff``: [ns, ns, 3] (a0 nm, alpha, beta) per species pair.  Displacements
    are per atom ([natoms, 3], nm) or, through ``to_sites``, per site as
    ``Structure.dsp``."""

    def __init__(self, st, vff):
        self.st = st
        self.vff = np.ascontiguousarray(vff, np.float64)
        self.ns = self.vff.shape[0]
        self.types = np.ascontiguousarray(st.types, dtype=np.uint8).reshape(-1)
        g = _Geom()
        g.nx, g.ny, g.nz = st.nx, st.ny, st.nz
        g.periodic[:] = [int(bool(x)) for x in st.periodic]
        g.lattice[:] = list(st.lattice)
        g.type = _p(self.types)
        g.dsp = None
        self._g = g
        ns = st.nsites
        slot = np.zeros(ns, np.int32)
        nbr = np.zeros(ns * 4, np.int32)
        wrap = np.zeros(ns * 12, np.int8)
        surf = np.zeros(ns, np.uint8)
        na = int(lib().orc_topology(C.byref(g), ns, _p(slot), _p(nbr), _p(wrap), _p(surf)))
        self.natoms = na
        self.atom_slot, self.nbr, self.surface = slot[:na].copy(), nbr[:na * 4].copy(), surf[:na].copy()

    def from_sites(self, dsp):
        if dsp is None:
            return np.zeros((self.natoms, 3))
        return np.asarray(dsp, np.float64).reshape(-1, 3)[self.atom_slot].copy()

    def to_sites(self, u):
        out = np.zeros((self.st.nsites, 3))
        out[self.atom_slot] = np.asarray(u).reshape(-1, 3)
        return out.reshape(self.st.nx, self.st.ny, self.st.nz, 8, 3)

    def energy(self, u):
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        grad = np.zeros_like(u)
        e = lib().orc_vff_energy(C.byref(self._g), self.natoms, _p(self.atom_slot), _p(self.nbr),
                                 self.ns, _p(self.vff), _p(u), _p(grad))
        return float(e), grad.reshape(-1, 3)

    def free_mask(self, bc):
        m = np.zeros(self.natoms, np.uint8)
        lib().orc_vff_free_mask(C.byref(self._g), self.natoms, _p(self.atom_slot),
                                _p(self.surface), int(bc), _p(m))
        return m.astype(bool)

    def relax(self, u0=None, bc=0, itmax=10000, tol=1e-9, end_if_small_step=1):
        u = np.ascontiguousarray(np.zeros((self.natoms, 3)) if u0 is None else u0,
                                 np.float64).reshape(-1).copy()
        e = np.zeros(1)
        its = lib().orc_vff_relax(C.byref(self._g), self.natoms, _p(self.atom_slot), _p(self.nbr),
                                  _p(self.surface), self.ns, _p(self.vff), int(bc), int(itmax),
                                  float(tol), int(end_if_small_step), _p(u), _p(e))
        return u.reshape(-1, 3), float(e[0]), int(its)
