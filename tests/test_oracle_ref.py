"""The oracle's Slater-Koster restatement against the reference's own routines.

``oracle/_ref/ref_sk`` links the reference's ``mb_ham_spds_micro.c`` compiled
from its own source (``oracle/build_ref.sh``).  These checks pin the parts of
the Hamiltonian that the golden eigenvalue files cannot: Harrison strain
scaling of the two-centre integrals, the strain diagonal correction, the
anion/cation orientation of the bond block, the spin-orbit on-site block and
the sp3s* -> sp3d5s* parameter conversion (mb_ham_spds_micro.c:597-1505,
2848-3026).  Skipped where neither the binary nor the reference tree exists.
"""

import os
import struct
import subprocess

import numpy as np
import pytest

from nemo3d_b200 import materials as M
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_sk")

# (material, nbasis passed to the reference, spin model, oracle norb, nspin)
MODELS = {
    "sp3d5s*_so": ("GaAs_spds", 20, 1, 10, 2),
    "sp3d5s*": ("GaAs_spds", 10, -1, 10, 1),
    "sp3s*_so": ("GaAs_sps", 10, 1, 5, 2),
}
# the four bond directions anion -> cation of a zincblende anion, in units of a
TETRA = np.array([[1, 1, 1], [-1, -1, 1], [1, -1, -1], [-1, 1, -1]], float) * 0.25


@pytest.fixture(scope="module")
def ref_sk():
    if not os.path.exists(REF_BIN):
        subprocess.check_call(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")])
    if not os.path.exists(REF_BIN):
        pytest.skip("reference sources not present; oracle/_ref/ref_sk not built")
    return REF_BIN


def _run(binary, payload: bytes) -> bytes:
    p = subprocess.run([binary], input=payload, capture_output=True, timeout=120)
    assert p.returncode == 0, p.stderr.decode()
    return p.stdout


def _cmat(buf, nb):
    a = np.frombuffer(buf, dtype=np.float64).reshape(nb, nb, 2)
    return a[..., 0] + 1j * a[..., 1]


def _bonds(rng, a0, count):
    out = []
    for i in range(count):
        nnv0 = TETRA[i % 4] * a0
        nnv = nnv0 * (1 + rng.normal(0, 0.02)) + rng.normal(0, 0.01 * a0, 3)
        out.append((nnv, nnv0))
    return out


@pytest.mark.parametrize("model", list(MODELS))
@pytest.mark.parametrize("with_strain", [1, 0])
def test_bond_blocks_and_strain_correction(ref_sk, model, with_strain):
    mat_name, nbasis, spin_model, norb, nspin = MODELS[model]
    rng = np.random.default_rng(7)
    for mname in (mat_name, mat_name.replace("GaAs", "InAs")):
        par = O.prepare_params(M.MATERIALS[mname], include_strain=True)
        a0 = par[31]
        payload = b""
        cases = []
        for this_cation in (0, 1):
            for nnv, nnv0 in _bonds(rng, a0, 8):
                payload += struct.pack("<5i", 1, nbasis, spin_model, this_cation, with_strain)
                payload += np.concatenate([nnv, nnv0, [a0], par[:35], par[35:]]).tobytes()
                cases.append((this_cation, nnv, nnv0))
        out = _run(ref_sk, payload)
        step = 2 * nbasis * nbasis * 16
        assert len(out) == step * len(cases)
        for i, (this_cation, nnv, nnv0) in enumerate(cases):
            ho = _cmat(out[i * step:i * step + step // 2], nbasis)
            hd = _cmat(out[i * step + step // 2:(i + 1) * step], nbasis)
            blk = np.zeros(norb * norb)
            ediag = np.zeros(norb)
            O.lib().orc_bond(norb, this_cation, O._p(np.ascontiguousarray(nnv)),
                             O._p(np.ascontiguousarray(nnv0)), O._p(par), with_strain,
                             float(a0), O._p(blk), O._p(ediag))
            blk = blk.reshape(norb, norb)            # [cation c][anion a]
            want = blk if not this_cation else blk.T  # rows: the neighbour's orbitals
            scale = np.abs(blk).max()
            assert np.abs(ho.imag).max() == 0.0
            assert np.abs(ho.real[:norb, :norb] - want).max() <= 1e-12 * scale, (mname, i)
            if nspin == 2:  # spin-down copy, no spin-flip hopping
                assert np.abs(ho.real[norb:, norb:] - want).max() <= 1e-12 * scale
                assert np.abs(ho[:norb, norb:]).max() == 0.0
                assert np.abs(ho[norb:, :norb]).max() == 0.0
            for half in range(nspin):  # the correction is the same for both spins
                corr = np.diag(hd.real)[half * norb:(half + 1) * norb]
                assert np.abs(corr - ediag).max() <= 1e-12 * max(1.0, np.abs(ediag).max()), \
                    (mname, i, half)
            if not with_strain:
                assert np.abs(ediag).max() == 0.0


@pytest.mark.parametrize("model", list(MODELS))
def test_onsite_block(ref_sk, model):
    mat_name, nbasis, spin_model, norb, nspin = MODELS[model]
    rng = np.random.default_rng(3)
    base = O.prepare_params(M.MATERIALS[mat_name], include_strain=True)[:35]
    payload = b""
    cases = []
    for cation in (0, 1):
        for _ in range(3):
            p = base + rng.normal(0, 0.05, 35)  # stands in for a bond average
            payload += struct.pack("<4i", 2, nbasis, spin_model, cation) + p.tobytes()
            cases.append((cation, p))
    out = _run(ref_sk, payload)
    step = nbasis * nbasis * 16
    for i, (cation, p) in enumerate(cases):
        h_ref = _cmat(out[i * step:(i + 1) * step], nbasis)
        h = np.zeros(nbasis * nbasis * 2)
        O.lib().orc_onsite_block(norb, nspin, cation, O._p(p), O._p(h))
        h = h.reshape(nbasis, nbasis, 2)
        assert np.array_equal(h[..., 0] + 1j * h[..., 1], h_ref), (model, cation)


def test_sp3s_parameter_conversion(ref_sk):
    for name in ("GaAs_sps", "InAs_sps"):
        mat = M.MATERIALS[name]
        pv = np.asarray(mat["pv"], float)[:15]
        out = _run(ref_sk, struct.pack("<i", 3) + pv.tobytes() + struct.pack("<d", mat["a0"]))
        ref = np.frombuffer(out, np.float64)
        ours = np.zeros(O.NPAR)
        O.lib().orc_prepare_params(1, 0, O._p(np.ascontiguousarray(pv)),
                                   O._p(np.zeros(O.NSTR)), 0.0, float(mat["a0"]), O._p(ours))
        assert np.array_equal(ours[:35], ref), name


@pytest.mark.parametrize("model,nbasis,norb", [("sp3d5s*_so", 20, 10), ("sp3s*_so", 10, 5)])
def test_dangling_bond_passivation(ref_sk, model, nbasis, norb):
    """The oracle's passivation of surface atoms against the reference's
    h3d_diag_dangling_bond_shift_zincblende (mb_ham_spds_micro.c:1910-2150),
    with the reference's own zincblende cell (Cell.c): a closed 3x3x3-cell
    GaAs box with random vacancies, so that faces, edges, corners and
    vacancy neighbours give every pattern of lost bonds and both signs of
    the last bond's direction.  The oracle's addition is its on-site block
    built with the passivation minus the block built without it (no strain
    shift, so the difference is the term alone up to one rounding of the
    diagonal)."""
    from nemo3d_b200 import workloads as W
    fam = ["GaAs_spds", "InAs_spds"] if norb == 10 else ["GaAs_sps", "InAs_sps"]
    mats = [M.MATERIALS[m] for m in fam]
    rng = np.random.default_rng(11)
    st = W.gaas_cube(3)
    t = st.types.reshape(-1).copy()
    t[rng.random(t.size) < 0.08] = 0  # vacancies
    st.types = t.reshape(st.types.shape)
    shift = 30.0
    on = O.OracleHamiltonian(st, norb, 2, mats, include_strain=False, passivate=True,
                             dangling_shift=shift)
    off = O.OracleHamiltonian(st, norb, 2, mats, include_strain=False, passivate=False)
    nb = 2 * norb
    dh = (on.onsite - off.onsite).reshape(on.natoms, nb, nb, 2)
    occ = np.zeros(st.nsites, np.uint8)
    occ[on.atom_slot] = 1  # the sites that hold an atom after the unbonded ones left
    pairs = np.stack([on.atom_slot // 8, on.atom_slot % 8], -1).astype(np.int32)
    payload = struct.pack("<5i", 4, nbasis, st.nx, st.ny, st.nz) + struct.pack("<d", shift)
    payload += occ.tobytes() + struct.pack("<i", len(pairs)) + pairs.tobytes()
    out = _run(ref_sk, payload)
    step = nbasis * nbasis * 16
    assert len(out) == step * len(pairs)
    patterns = set()
    nsurf = 0
    for a in range(on.natoms):
        ref = _cmat(out[a * step:(a + 1) * step], nbasis)
        got = dh[a, ..., 0] + 1j * dh[a, ..., 1]
        if on.surface[a]:
            nsurf += 1
            patterns.add(tuple(on.nbr[4 * a:4 * a + 4] >= 0))
            # 1e-15 relative to the shift, one rounding of a ~10 eV diagonal
            assert np.abs(got - ref).max() <= 2e-15 * shift, (a, np.abs(got - ref).max())
        else:  # four bonds: nothing to passivate, in either code
            assert np.abs(ref).max() == 0.0 and np.abs(got).max() == 0.0
    assert nsurf > 100
    assert len(patterns) >= 10, patterns  # most of the 15 bond-loss patterns occur


@pytest.mark.parametrize("case", ["cube_sp3s", "dome_spds_so"])
def test_oracle_lanczos_matches_reference_lanczos(case):
    """The oracle's restatement of the Lanczos driver (oracle/tb_oracle.c)
    against the reference's own eigenvaluesLanczos (eigen/src/lanczos.c,
    compiled from its source into oracle/_ref/libref_lanczos.so), both on
    the oracle's H*x: the same eigenvalues (1e-10 eV) and iteration count;
    the iteration at which each value was accepted agrees to one check
    interval (the inverse iterations of the test start from a seeded
    generator here and from glibc rand() there, which can move a borderline
    acceptance by one check)."""
    from nemo3d_b200 import workloads as W
    if not O.ref_lanczos_available():
        pytest.skip("oracle/_ref/libref_lanczos.so not built (reference sources absent)")
    if case == "cube_sp3s":
        st = W.gaas_cube(4)
        o = O.OracleHamiltonian(st, 5, 1, [M.MATERIALS["GaAs_sps"], M.MATERIALS["InAs_sps"]])
        kw = dict(imax=3000, req=(3, 3), erange1=(-0.5, 0.0), erange2=(1.5, 2.5))
    else:
        st = W.dome_in_box(cells=(5, 5, 4), base_nm=1.8, height_nm=0.8, wl_z_nm=0.6,
                           sigma_frac=0.01, seed=4)
        o = O.OracleHamiltonian(st, 10, 2, [M.MATERIALS["GaAs_spds"], M.MATERIALS["InAs_spds"]])
        kw = dict(imax=2500, req=(2, 2), erange1=(-0.6, 0.75), erange2=(1.5, 2.8))
    r0 = W.random_start(o.n, seed=0)
    kw.update(tol=1e-7, conv_start=100, conv_skip=50)
    ref = O.ref_eigenvalues_lanczos(o, r0, **kw)
    got = o.lanczos(r0, **kw)
    assert len(ref["evals"]) == len(got["evals"]) >= 2
    assert np.abs(ref["evals"] - got["evals"]).max() < 1e-10
    assert ref["iterations"] == got["iterations"]
    assert np.abs(ref["conv_it"] - got["conv_it"]).max() <= kw["conv_skip"]


@pytest.mark.parametrize("model,cube,p,skip", [("sp3s*", 3, 3, 10), ("sp3s*_so", 2, 4, 20),
                                               ("sp3d5s*_so", 2, 8, 10)])
def test_oracle_block_lanczos_matches_reference(model, cube, p, skip):
    """The oracle's restatement of the block Lanczos (oracle.block_lanczos)
    against the reference's own block_Lanczos_QR + block_lanczos_blocktridiagonal
    (eigen/src/lanczos_blk.c, compiled from its source into
    oracle/_ref/libref_lanczos.so), both on the oracle's H*x from the same
    start block: the same number of block steps and of values found, each
    value within the convergence tolerance (1e-7 eV: the Method-4 test
    accepts a value once it moved less than that between two checks, and the
    value reported is the one at that check).  Both the lowest and the
    highest part of the spectrum are searched through the reference's second
    window (its first reads one entry past zhbevx's values)."""
    if not O.ref_lanczos_available():
        pytest.skip("oracle/_ref/libref_lanczos.so not built (reference sources absent)")
    from nemo3d_b200 import workloads as W
    fam = "spds" if model.startswith("sp3d5s") else "sps"
    norb, nspin = M.BAND_MODELS[model]
    o = O.OracleHamiltonian(W.gaas_cube(cube), norb, nspin, [M.MATERIALS[f"GaAs_{fam}"]])
    ev = np.linalg.eigvalsh(o.dense())
    r0 = np.random.default_rng(11).uniform(-1, 1, size=(p, 2 * o.n))

    def hx(q):
        y = o.hx(np.column_stack([q.real, q.imag]).ravel())
        return y[0::2] + 1j * y[1::2]

    for win in ((ev[0] - 0.5, ev[0] + 1.0), (ev[-1] - 1.0, ev[-1] + 0.5)):
        kw = dict(imax=min(300, o.n // p - 2), req=(0, 3), erange1=(0.0, 0.0), erange2=win,
                  tol=1e-7, conv_start=30, conv_skip=skip)
        ref = O.ref_block_lanczos(o, r0, **kw)
        got = O.block_lanczos(hx, r0, **kw)
        assert (ref["found_vb"], ref["found_cb"]) == (got["found_vb"], got["found_cb"]) == (0, 3)
        assert ref["iterations"] == got["iterations"]
        assert np.abs(np.sort(ref["evals"]) - np.sort(got["evals"])).max() < 1e-7
