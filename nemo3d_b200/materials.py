"""Tight-binding material parameter sets and species numbering.

The numbers below are the parameter sets shipped with NEMO-3D in
``NEMO_3D/XMLtoC/xml/ioNemo3D.xml`` (``mb_pv``: 35 two-centre/on-site
parameters for sp3d5s*, or 15 for sp3s*; ``mb_strain``: 33 strain exponents,
energy shifts and strain-correction coefficients; ``Ev_offset``).  They are data,
not code: a Hamiltonian can only agree with the reference's when it is built
from the same numbers, so they are carried over verbatim and each set names the
XML line it comes from.

Species are numbered here (``SPECIES``); 0 means "no atom" in an atom-type grid.
The cation/anion role of an atom is fixed by its zincblende sub-lattice (in-cell
sites 0..3 are cations, 4..7 anions), as in ``geo_struct::isCation``.
"""

from __future__ import annotations

# species numbering used in atom-type grids (0 = empty site)
SPECIES = {"Ga": 1, "In": 2, "Al": 3, "As": 4, "Si": 5, "Ge": 6}

# band models, named as in mb_ham_spds_micro2.h (BM_Type)
BAND_MODELS = {
    # name: (orbitals per spin, spins)
    "sp3s*": (5, 1),             # spin-up block of Bands_10_sp3ss_spin with SO = 0
    "sp3s*_so": (5, 2),          # Bands_10_sp3ss_spin
    "sp3d5s*": (10, 1),          # Bands_10_sp3d5ss_nospin
    "sp3d5s*_so": (10, 2),       # Bands_20_sp3d5ss_spin
}

SP3D5S = "sp3d5s*"
SP3S = "sp3s*"

# name -> dict(cation, anion, family, a0 [nm], pv, strain, ev_offset, source)
MATERIALS = {
    "GaAs_spds": dict(
        cation="Ga", anion="As", family=SP3D5S, a0=0.56532, ev_offset=0.0,
        source="ioNemo3D.xml:577-724",
        pv=[-5.50042, 4.15107, -0.24119, 6.70776, 19.71059, 22.66352, 13.03169,
            12.74846, 0.17234, 0.02179, -1.64508, -3.704550, -2.20777, -1.31491,
            2.66493, 2.96032, 1.97650, 1.02755, -2.609400, -2.32059, -0.62820,
            0.13324, 4.15080, -1.42744, -1.87428, -1.88964, 2.52926, 2.54913,
            -1.26996, 2.50536, -0.85174, 0.56532, 1, 1, 1],
        strain=[0.00000, 0.21266, 2.06001, 1.38498, 2.68497, 1.31405, 1.89889,
                1.39930, 1.81235, 2.37964, 2.93686, 1.72443, 1.97253, 1.89672,
                1.78540, 27.0, 27.0, 0.58696, 0.48609, 0.88921, 0.77095, 0.75979,
                1.45891, 0.81079, 1.21202, 1.07015, 0.38053, 1.03256, 1.32385,
                2.00000, 1.61350, 1.50000, 1.26262]),
    "InAs_spds": dict(
        cation="In", anion="As", family=SP3D5S, a0=0.60583, ev_offset=0.0,
        source="ioNemo3D.xml:728-875",
        pv=[-5.50042, 4.15107, -0.581930, 6.97163, 19.71059, 19.94138, 13.03169,
            13.30709, 0.17234, 0.139670, -1.69435, -4.21045, -2.42674, -1.159870,
            2.598230, 2.809360, 2.06766, 0.93734, -2.26837, -2.293090, -0.899370,
            -0.488990, 4.310640, -1.288950, -1.731410, -1.978420, 2.188860,
            2.456020, -1.584610, 2.71793, -0.505090, 0.60583, 1, 1, 1],
        strain=[0.060800, 0.000810, 1.92494, 1.570030, 2.06151, 1.602470,
                1.765660, 1.949370, 2.383820, 2.455600, 1.94235, 2.32291, 1.84572,
                2.3296, 2.02387, 27.0, 27.0, 1.258286, 2.481447, 1.086223,
                4.557774, 4.367575, 7.02966, 3.298598, 7.029496, 0.0000, 0.187036,
                1.195042, 1.769483, 4.624483, 0.0000, 0.0000, 0.246999]),
    "Si_spds": dict(
        cation="Si", anion="Si", family=SP3D5S, a0=0.543095, ev_offset=0.0,
        source="ioNemo3D.xml:1030-1184",
        pv=[-2.15168, 4.22925, -2.15168, 4.22925, 19.11650, 19.11650, 13.78950,
            13.78950, 0.01989, 0.01989, -1.95933, -4.24135, -1.52230, -1.52230,
            3.02562, 3.02562, 3.15565, 3.15565, -2.28485, -2.28485, -0.80993,
            -0.80993, 4.10364, -1.51801, -1.35554, -1.35554, 2.38479, 2.38479,
            -1.68136, 2.58880, -1.81400, 0.543095, 1, 1, 1],
        strain=[0.13203, 0.19237, 0.56247, 2.36548, 0.49435, 1.84385, 2.5672,
                0.34492, 2.23636, 4.5125, 2.00203, 4.66836, 2.30238, 0.92391,
                1.08601, 27, 27, 0.83942, 0.38885, 0.89216, 0.89216, 0.24004,
                0.24004, 1.7944, 1.7944, 0, 0, 0.17104, 0.17104, 2.0332, 0, 0,
                2.64866]),
    "GaAs_sps": dict(
        cation="Ga", anion="As", family=SP3S, a0=0.56532, ev_offset=0.0,
        source="ioNemo3D.xml:1658-1803",
        pv=[-8.5107, 0.954046, -2.77475, 3.43405, 8.45405, 6.58405, -6.4513,
            1.9546, 4.77, 4.68, 7.7, 4.85, 7.01, 0.42, 0.174],
        strain=[2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 0, 27.0, 27.0, 1, 1, 1,
                1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0]),
    "InAs_sps": dict(
        cation="In", anion="As", family=SP3S, a0=0.60583, ev_offset=0.227948,
        source="ioNemo3D.xml:1804-1946",
        pv=[-9.60889, 0.739114, -2.55269, 3.71931, 7.40911, 6.73931, -5.4052,
            1.8398, 4.4693, 3.0354, 6.3389, 3.3744, 3.9097, 0.42, 0.393],
        strain=[2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 0, 27.0, 27.0, 1, 1, 1,
                1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0]),
}


# Keating valence-force-field constants per (cation, anion) compound: the
# unstrained cubic cell length a0 (nm) and alpha, beta (the strain_alpha and
# strain_beta entries of the same XML material blocks; strain3d.c reads them
# through StrainParam::amat/alpha/beta).
VFF = {
    ("Ga", "As"): dict(a0=0.56532, alpha=41.49, beta=8.94, source="ioNemo3D.xml:658-673"),
    ("In", "As"): dict(a0=0.60583, alpha=35.18, beta=5.49, source="ioNemo3D.xml:809-824"),
    ("Si", "Si"): dict(a0=0.543095, alpha=48.5, beta=13.8, source="ioNemo3D.xml:1111-1126"),
}


def vff_table(pairs=None, nspecies=8):
    """[nspecies, nspecies, 3] table (a0, alpha, beta) for the compounds in
    ``pairs`` (default: all of ``VFF``), symmetric in the two species."""
    import numpy as np
    t = np.zeros((nspecies, nspecies, 3))
    for (c, a) in (pairs or VFF):
        v = VFF[(c, a)]
        t[SPECIES[c], SPECIES[a]] = t[SPECIES[a], SPECIES[c]] = (v["a0"], v["alpha"], v["beta"])
    return t


def material_family(model: str) -> str:
    """Parameter family a band model draws on ("sp3s*" or "sp3d5s*")."""
    return SP3S if model.startswith("sp3s*") else SP3D5S


def materials_for(model: str, names=None):
    """Material sets usable with ``model`` (all of its family unless named)."""
    fam = material_family(model)
    sel = [n for n in (names or MATERIALS) if MATERIALS[n]["family"] == fam]
    if not sel:
        raise ValueError(f"no material set of family {fam} among {names}")
    return [MATERIALS[n] for n in sel]
