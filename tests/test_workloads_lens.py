"""The warm start's training distribution (workloads.lens_dot, random_lens),
on CPU.

Bars: the same seed gives the same structure; the lens and its wetting
layer hold In only on cation sites and only where the shape says (the
anions stay As); the In fraction of the lens follows x_in; random_lens
draws its parameters inside the stated ranges.
"""
import numpy as np

from nemo3d_b200 import workloads
from nemo3d_b200.materials import SPECIES


def test_lens_dot_is_seeded_and_shaped():
    a = workloads.lens_dot((14, 14, 10), base_nm=4.0, height_nm=1.5, x_in=0.6,
                           center=(0.4, 0.6), seed=7)
    b = workloads.lens_dot((14, 14, 10), base_nm=4.0, height_nm=1.5, x_in=0.6,
                           center=(0.4, 0.6), seed=7)
    assert np.array_equal(a.types, b.types) and np.array_equal(a.dsp, b.dsp)
    assert (a.types[..., 4:] == SPECIES["As"]).all()
    cat = a.types[..., :4]
    assert set(np.unique(cat)) <= {SPECIES["Ga"], SPECIES["In"]}
    # In only inside the lens or the one-monolayer wetting layer
    pos = a.site_positions()[..., :4, :]
    lat = a.lattice[0]
    z0 = 0.3 * a.nz * lat
    cx, cy = 0.4 * a.nx * lat - 0.5 * lat, 0.6 * a.ny * lat - 0.5 * lat
    wl = (pos[..., 2] >= z0 - 0.5 * lat) & (pos[..., 2] < z0)
    lens = (pos[..., 2] >= z0) & (((pos[..., 0] - cx) / 2.0) ** 2 + ((pos[..., 1] - cy) / 2.0) ** 2
                                  + ((pos[..., 2] - z0) / 1.5) ** 2 <= 1.0)
    inside = wl | lens
    assert not (cat[~inside] == SPECIES["In"]).any()
    frac = (cat[inside] == SPECIES["In"]).mean()
    assert abs(frac - 0.6) < 0.1


def test_random_lens_ranges():
    for s in range(20):
        info = workloads.random_lens(s).info
        assert 4.0 <= info["base_nm"] <= 7.0 and 1.5 <= info["height_nm"] <= 3.0
        assert 0.4 <= info["x_in"] <= 1.0
        assert all(0.25 <= c <= 0.75 for c in info["center"])
    assert workloads.random_lens(3).info == workloads.random_lens(3).info
