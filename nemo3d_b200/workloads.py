"""Synthetic zincblende structures with the shapes of the benchmark configurations.

A structure is a dense grid of conventional cubic cells (cell (i,j,k) row-major,
k fastest -- the order in which ``geo_struct::FillFirstShape``
(base/ham3d.c:745-900) enumerates cells) with eight sites per cell (sites 0..3
cations, 4..7 anions, positions from ``Cell::Initialize``, base/Cell.c:185-210).
Each site holds a species id (``materials.SPECIES``, 0 = empty) and optionally
a displacement in nm, the seam through which the reference receives strain
(``geo_struct::l_m_2_atomdsp``, base/geo_struct.c:2224-2297).

These generators stand in for the reference's XML shape decks and its Keating
strain solver, which are out of scope; they are inputs, not parity targets.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .materials import SPECIES

# in-cell site positions in units of the lattice constant (Cell.c:185-210)
SITE_POS = np.array([
    [0, 0, 0], [0, -0.5, -0.5], [-0.5, -0.5, 0], [-0.5, 0, -0.5],
    [-0.25, -0.25, -0.25], [-0.25, -0.75, -0.75], [-0.75, -0.75, -0.25],
    [-0.75, -0.25, -0.75]], dtype=np.float64)

A_GAAS = 0.56532  # GaAs lattice constant of the shipped parameter set (nm)


@dataclass
class Structure:
    nx: int
    ny: int
    nz: int
    lattice: tuple = (A_GAAS, A_GAAS, A_GAAS)
    periodic: tuple = (False, False, False)
    types: np.ndarray = None          # uint8 [nx, ny, nz, 8]
    dsp: np.ndarray | None = None     # float64 [nx, ny, nz, 8, 3] (nm) or None
    name: str = ""
    info: dict = field(default_factory=dict)

    @property
    def nsites(self) -> int:
        return self.nx * self.ny * self.nz * 8

    def site_positions(self) -> np.ndarray:
        """Unstrained site positions (nm), shape [nx, ny, nz, 8, 3]."""
        ijk = np.stack(np.meshgrid(np.arange(self.nx), np.arange(self.ny),
                                   np.arange(self.nz), indexing="ij"), -1)
        pos = ijk[:, :, :, None, :] + SITE_POS[None, None, None]
        return pos * np.asarray(self.lattice)


def _binary(nx, ny, nz, cation="Ga", anion="As"):
    t = np.zeros((nx, ny, nz, 8), dtype=np.uint8)
    t[..., :4] = SPECIES[cation]
    t[..., 4:] = SPECIES[anion]
    return t


def bulk_cell(cation="Ga", anion="As", a=A_GAAS) -> Structure:
    """One periodic conventional cell (the reference's bulk decks)."""
    return Structure(1, 1, 1, (a, a, a), (True, True, True),
                     _binary(1, 1, 1, cation, anion), None, f"{cation}{anion}_bulk")


def gaas_cube(n: int = 8, a: float = A_GAAS) -> Structure:
    """Closed GaAs cube of n x n x n conventional cells (4096 atoms for n=8)."""
    return Structure(n, n, n, (a, a, a), (False, False, False),
                     _binary(n, n, n), None, f"GaAs_cube_{n}")


def dome_in_box(cells=(58, 58, 38), base_nm: float = 20.0, height_nm: float = 5.0,
                wl_z_nm: float | None = None, sigma_frac: float = 0.005,
                seed: int = 1, a: float = A_GAAS) -> Structure:
    """InAs lens (dome) on a one-monolayer InAs wetting layer in a GaAs box.

    The dome is the half-ellipsoid of ``isNotInDome`` (base/ham3d.c:233-256):
    centred in x,y on the wetting layer, semi-axes base/2, base/2, height.
    Displacements are i.i.d. Gaussian per component with sigma equal to
    ``sigma_frac`` times the ideal GaAs bond length, drawn from ``seed``
    (a stand-in for the Keating strain field).
    """
    nx, ny, nz = cells
    t = _binary(nx, ny, nz)
    st = Structure(nx, ny, nz, (a, a, a), (False, False, False), t, None,
                   f"InAs_dome_{nx}x{ny}x{nz}")
    pos = st.site_positions()
    lx, ly, lz = nx * a, ny * a, nz * a
    z0 = wl_z_nm if wl_z_nm is not None else 0.3 * lz
    cx, cy = 0.5 * lx - 0.5 * a, 0.5 * ly - 0.5 * a
    cat = pos[..., :4, :]
    # wetting layer: the cation plane(s) within one monolayer (a/2) below z0
    wl = (cat[..., 2] >= z0 - 0.5 * a) & (cat[..., 2] < z0)
    rb, h = 0.5 * base_nm, height_nm
    dome = (cat[..., 2] >= z0) & (((cat[..., 0] - cx) / rb) ** 2 +
                                  ((cat[..., 1] - cy) / rb) ** 2 +
                                  ((cat[..., 2] - z0) / h) ** 2 <= 1.0)
    sub = t[..., :4]
    sub[wl | dome] = SPECIES["In"]
    if sigma_frac > 0:
        rng = np.random.default_rng(seed)
        sigma = sigma_frac * np.sqrt(3.0) / 4.0 * a
        st.dsp = rng.normal(0.0, sigma, size=(nx, ny, nz, 8, 3))
    st.info = dict(base_nm=base_nm, height_nm=height_nm, wl_z_nm=z0,
                   sigma_nm=sigma_frac * np.sqrt(3.0) / 4.0 * a, seed=seed,
                   n_in=int((sub == SPECIES["In"]).sum()))
    return st


def random_start(n_complex: int, seed: int = 0) -> np.ndarray:
    """Start vector with real and imaginary parts uniform in [-1, 1]."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=2 * n_complex)


def alloy_dot(natoms: int, x_in: float, seed: int = 0, a: float = A_GAAS) -> Structure:
    """Free-standing In(x)Ga(1-x)As nanocrystal of about ``natoms`` atoms: a
    box of cells as close to a cube as the count allows, every cation site In
    with probability ``x_in`` (independent per site, seeded), anions As; the
    surface is passivated by the Hamiltonian's dangling-bond shift."""
    ncell = max(1, int(round(natoms / 8)))
    n = max(1, int(round(ncell ** (1.0 / 3.0))))
    nz = max(1, int(round(ncell / (n * n))))
    rng = np.random.default_rng(seed)
    t = _binary(n, n, nz)
    t[..., :4] = np.where(rng.random((n, n, nz, 4)) < x_in, SPECIES["In"], SPECIES["Ga"])
    return Structure(n, n, nz, (a, a, a), (False, False, False), t, None,
                     f"InGaAs_dot_{n}x{n}x{nz}", dict(x_in=x_in, seed=seed))


def pack_dots(dots, gap: int = 1):
    """Place dots side by side along x in one grid, ``gap`` empty cells apart,
    so that no bond joins two of them (the Hamiltonian of the packed grid is
    block diagonal).  All dots must share the lattice constants.  Returns the
    packed structure and the cell boundaries along x ([ndots + 1]): dot d owns
    cells [bounds[d], bounds[d + 1]), its trailing gap included."""
    lat = dots[0].lattice
    if any(tuple(d.lattice) != tuple(lat) for d in dots):
        raise ValueError("packed dots must share the lattice constants")
    ny = max(d.ny for d in dots)
    nz = max(d.nz for d in dots)
    nx = sum(d.nx + gap for d in dots)
    t = np.zeros((nx, ny, nz, 8), np.uint8)
    dsp = None
    if any(d.dsp is not None for d in dots):
        dsp = np.zeros((nx, ny, nz, 8, 3))
    bounds = [0]
    x0 = 0
    for d in dots:
        t[x0:x0 + d.nx, :d.ny, :d.nz] = d.types
        if dsp is not None and d.dsp is not None:
            dsp[x0:x0 + d.nx, :d.ny, :d.nz] = d.dsp
        x0 += d.nx + gap
        bounds.append(x0)
    st = Structure(nx, ny, nz, tuple(lat), (False, False, False), t, dsp,
                   f"packed_{len(dots)}_dots", dict(ndots=len(dots)))
    return st, np.asarray(bounds, np.int32)


def lens_dot(cells=(20, 20, 14), base_nm: float = 6.0, height_nm: float = 2.0,
             x_in: float = 0.8, center=(0.5, 0.5), wl_z_frac: float = 0.3,
             sigma_frac: float = 0.005, seed: int = 0, a: float = A_GAAS) -> Structure:
    """In(x)Ga(1-x)As lens on a one-monolayer wetting layer of the same alloy
    in a GaAs box: the half-ellipsoid of ``dome_in_box`` with its axis at the
    fractional position ``center`` of the box in x, y, every cation site of
    the lens and the layer In with probability ``x_in`` (independent per
    site), Gaussian displacements as in ``dome_in_box``; all draws from
    ``seed``.  The randomized dots the learned warm start is trained on."""
    nx, ny, nz = cells
    rng = np.random.default_rng(seed)
    t = _binary(nx, ny, nz)
    st = Structure(nx, ny, nz, (a, a, a), (False, False, False), t, None,
                   f"InGaAs_lens_{nx}x{ny}x{nz}_s{seed}")
    pos = st.site_positions()
    z0 = wl_z_frac * nz * a
    cx, cy = center[0] * nx * a - 0.5 * a, center[1] * ny * a - 0.5 * a
    cat = pos[..., :4, :]
    wl = (cat[..., 2] >= z0 - 0.5 * a) & (cat[..., 2] < z0)
    rb, h = 0.5 * base_nm, height_nm
    lens = (cat[..., 2] >= z0) & (((cat[..., 0] - cx) / rb) ** 2 +
                                  ((cat[..., 1] - cy) / rb) ** 2 +
                                  ((cat[..., 2] - z0) / h) ** 2 <= 1.0)
    sub = t[..., :4]
    alloy = rng.random(sub.shape) < x_in
    sub[(wl | lens) & alloy] = SPECIES["In"]
    if sigma_frac > 0:
        sigma = sigma_frac * np.sqrt(3.0) / 4.0 * a
        st.dsp = rng.normal(0.0, sigma, size=(nx, ny, nz, 8, 3))
    st.info = dict(base_nm=base_nm, height_nm=height_nm, x_in=x_in, center=tuple(center),
                   seed=seed, n_in=int((sub == SPECIES["In"]).sum()))
    return st


def random_lens(seed: int, cells=(20, 20, 14)) -> Structure:
    """One draw of the warm start's training distribution: base 4-7 nm,
    height 1.5-3 nm, x_in uniform in [0.4, 1.0], lens axis uniform in the
    middle half of the box (all from ``seed``)."""
    rng = np.random.default_rng(10_000 + seed)
    base = rng.uniform(4.0, 7.0)
    height = rng.uniform(1.5, 3.0)
    x_in = rng.uniform(0.4, 1.0)
    center = tuple(rng.uniform(0.25, 0.75, 2))
    return lens_dot(cells, base, height, x_in, center, seed=seed)
