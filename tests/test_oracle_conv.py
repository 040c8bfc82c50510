"""The warm-start network's CPU oracle (oracle/conv_oracle.py) against
finite differences and direct counts.

Bars: convolution gradients (input, weights, bias) and the loss gradient
within 1e-7 relative of central differences in float64; bf16 rounding equal
to round-to-nearest-even of the float32 bits; features equal to a direct
per-voxel count; the start vector equal to its per-atom definition.
"""
import numpy as np
import pytest

import conv_oracle as co


def _fd(f, x, eps=1e-6):
    g = np.zeros_like(x)
    it = np.nditer(x, flags=["multi_index"])
    for _ in it:
        i = it.multi_index
        x0 = x[i]
        x[i] = x0 + eps
        fp = f()
        x[i] = x0 - eps
        fm = f()
        x[i] = x0
        g[i] = (fp - fm) / (2 * eps)
    return g


@pytest.mark.parametrize("relu", [False, True])
def test_conv_gradients_match_finite_differences(relu):
    rng = np.random.default_rng(1)
    n, cin, cout, G = 2, 2, 3, 4
    x = rng.normal(size=(n, cin, G, G, G))
    w = co.bf16_round(rng.normal(size=(cout, cin, 27)).astype(np.float32))
    b = rng.normal(size=cout)
    r = rng.normal(size=(n, cout, G, G, G))

    def f():
        return float((co.conv3d_fwd(x, w, b, relu) * r).sum())

    out = co.conv3d_fwd(x, w, b, relu)
    g = r * (out > 0) if relu else r
    dx, dw, db = co.conv3d_bwd(x, w, g)
    for got, var in ((dx, x), (dw, w), (db, b)):
        want = _fd(f, var)
        assert np.abs(got - want).max() <= 1e-7 * max(1.0, np.abs(want).max())


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    n, k, G = 3, 4, 3
    out = rng.normal(size=(n, k + 1, G, G, G))
    env = rng.normal(size=(n, k, G, G, G))
    sig = rng.normal(size=n)
    _, d, sp = co.loss(out, env, sig, 0.7)
    assert np.allclose(sp, out[:, k].reshape(n, -1).mean(1))
    want = _fd(lambda: co.loss(out, env, sig, 0.7)[0], out)
    assert np.abs(d - want).max() <= 1e-8


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.14159, 1e-3], np.float32)
    r = co.bf16_round(vals)
    for v, got in zip(vals, r):
        lo = np.float32(np.frombuffer(np.uint32(np.float32(v).view(np.uint32) & 0xFFFF0000).tobytes(),
                                      np.float32)[0])
        step = np.spacing(np.float32(abs(lo))) * 2 ** 16
        hi = lo + np.sign(v) * step
        assert got in (lo, hi)
        assert abs(got - v) <= abs(v - (hi if got == lo else lo)) + 1e-12
    assert co.bf16_round(np.float32(1.00390625)) == 1.0  # tie -> even


def test_features_direct_count():
    from nemo3d_b200 import materials, workloads
    st = workloads.lens_dot((6, 5, 4), base_nm=2.0, height_nm=1.0, x_in=0.7, seed=3)
    G = 3
    f = co.features(st.types, st.dsp, G, materials.SPECIES["In"])
    for v in range(G ** 3):
        vx, vy, vz = v // (G * G), (v // G) % G, v % G
        cells = [(i, j, k) for i in range(st.nx) for j in range(st.ny) for k in range(st.nz)
                 if (i * G) // st.nx == vx and (j * G) // st.ny == vy and (k * G) // st.nz == vz]
        t = np.array([st.types[c] for c in cells]) if cells else np.zeros((0, 8))
        ncat = (t[:, :4] > 0).sum()
        nin = (t[:, :4] == materials.SPECIES["In"]).sum()
        assert f[0, v] == pytest.approx(nin / ncat if ncat else 0.0)
        occ = t > 0
        assert f[1, v] == pytest.approx(occ.sum() / t.size if t.size else 0.0)
        if occ.sum():
            d = np.array([np.linalg.norm(st.dsp[c], axis=-1) for c in cells])
            assert f[2, v] == pytest.approx(d[occ].mean() * 1000.0)


def test_start_vector_definition():
    rng = np.random.default_rng(4)
    dims, nb, G, k = (3, 2, 2), 4, 2, 2
    sites = np.array([0, 5, 8 * 3 + 1, 8 * 7 + 6, 8 * 11 + 4])
    env = rng.random((k, G ** 3))
    prof = rng.random((k, 2, nb))
    u = rng.uniform(-1, 1, sites.size * nb) + 1j * rng.uniform(-1, 1, sites.size * nb)
    r = co.start_vector(sites, dims, nb, env, prof, G, 0.01, u)
    for a, s in enumerate(sites):
        cell, m = s >> 3, s & 7
        kk, jj, ii = cell % 2, (cell // 2) % 2, cell // 4
        v = ((ii * G) // 3 * G + (jj * G) // 2) * G + (kk * G) // 2
        for o in range(nb):
            w2 = 0.01 + sum(env[q, v] ** 2 * prof[q, int(m >= 4), o] for q in range(k))
            assert r[a * nb + o] == pytest.approx(u[a * nb + o] * np.sqrt(w2))
