"""Learned warm start on the GPU: the network kernels against the CPU
oracle, training, and the warm solve against the cold one.

Bars: convolution forward and both backward kernels within 2e-5 of the
largest magnitude of the oracle's float64 result on the same bf16 weights
(float accumulation); loss, sigma and gradient within 1e-5 relative; Adam
within 1e-6 relative and the bf16 copy equal to the rounded master weights;
features exact for the counts and within 1e-5 for the displacement proxy;
the start vector within 1e-6 relative; a network-level gradient (4 layers)
against the oracle's chain within 1e-4 relative; training lowers the loss
on a fixed batch; the warm solve finds the cold solve's 8 levels within
1e-6 eV, and with no network it is the cold solve.
"""
import numpy as np
import pytest

import conv_oracle as co
from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype or torch.float32).cuda()


def _conv_case(n, cin, cout, G, relu, seed):
    import torch
    from nemo3d_b200 import warmstart as ws
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, cin, G ** 3)).astype(np.float32)
    w32 = rng.normal(size=(cout, cin, 27)).astype(np.float32) * 0.2
    b = rng.normal(size=cout).astype(np.float32)
    wbits = co.bf16_bits(w32)
    wq = co.bf16_round(w32)
    X, W, B = _t(x), _t(wbits.view(np.int16), torch.int16), _t(b)
    out = torch.empty((n, cout, G ** 3), device="cuda")
    assert ws._lib().tbgpu_ws_conv3d_fwd(ws._ptr(X), ws._ptr(W), ws._ptr(B), ws._ptr(out), n, cin,
                                        cout, G, int(relu)) == 0
    x5 = x.astype(np.float64).reshape(n, cin, G, G, G)
    want = co.conv3d_fwd(x5, wq, b.astype(np.float64), relu)
    return X, W, out, x5, wq, want, rng


@pytest.mark.parametrize("n,cin,cout,G,relu", [(2, 3, 32, 6, True), (3, 32, 9, 5, False),
                                               (1, 32, 32, 8, True), (2, 5, 11, 4, True)])
def test_conv_kernels_match_oracle(n, cin, cout, G, relu):
    import torch
    from nemo3d_b200 import warmstart as ws
    X, W, out, x5, wq, want, rng = _conv_case(n, cin, cout, G, relu, seed=cin + cout)
    got = out.cpu().numpy().reshape(want.shape)
    assert np.abs(got - want).max() <= 2e-5 * np.abs(want).max()
    dout = rng.normal(size=want.shape).astype(np.float32)
    g = dout * (want > 0) if relu else dout.astype(np.float64)
    dx, dw, db = co.conv3d_bwd(x5, wq, g)
    D = _t(dout.reshape(n, cout, -1))
    act = out if relu else None
    din = torch.empty_like(X)
    gw = torch.empty((cout, cin, 27), device="cuda")
    gb = torch.empty(cout, device="cuda")
    assert ws._lib().tbgpu_ws_conv3d_bwd_data(ws._ptr(D), ws._ptr(act), ws._ptr(W), ws._ptr(din),
                                             n, cin, cout, G) == 0
    assert ws._lib().tbgpu_ws_conv3d_bwd_weight(ws._ptr(X), ws._ptr(D), ws._ptr(act), ws._ptr(gw),
                                               ws._ptr(gb), n, cin, cout, G) == 0
    for got, ref in ((din, dx), (gw, dw), (gb, db)):
        got = got.cpu().numpy().reshape(ref.shape)
        assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max()


def test_loss_and_adam_match_oracle():
    import torch
    from nemo3d_b200 import warmstart as ws
    rng = np.random.default_rng(3)
    n, k, G = 3, 8, 5
    out = rng.normal(size=(n, k + 1, G ** 3)).astype(np.float32)
    env = rng.normal(size=(n, k, G ** 3)).astype(np.float32)
    sig = rng.normal(size=n).astype(np.float32)
    O, E, S = _t(out), _t(env), _t(sig)
    d = torch.empty_like(O)
    sp = torch.empty(n, device="cuda")
    ls = torch.empty(1, device="cuda")
    assert ws._lib().tbgpu_ws_loss(ws._ptr(O), ws._ptr(E), ws._ptr(S), n, k, G, 0.5, ws._ptr(d),
                                  ws._ptr(sp), ws._ptr(ls)) == 0
    L, dref, spref = co.loss(out.astype(np.float64).reshape(n, k + 1, G, G, G),
                             env.astype(np.float64).reshape(n, k, G, G, G), sig, 0.5)
    assert ls.item() == pytest.approx(L, rel=1e-5)
    assert np.allclose(sp.cpu().numpy(), spref, rtol=1e-5, atol=1e-6)
    assert np.abs(d.cpu().numpy() - dref.reshape(n, k + 1, -1)).max() <= 1e-5 * np.abs(dref).max()
    # Adam, three steps
    w = rng.normal(size=1000).astype(np.float32)
    Wt, Wb = _t(w), torch.empty(1000, dtype=torch.int16, device="cuda")
    M, V = torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    wr, mr, vr = w.astype(np.float64), np.zeros(1000), np.zeros(1000)
    for step in (1, 2, 3):
        g = rng.normal(size=1000).astype(np.float32)
        assert ws._lib().tbgpu_ws_adam(ws._ptr(Wt), ws._ptr(Wb), ws._ptr(_t(g)), ws._ptr(M),
                                      ws._ptr(V), 1000, 1e-2, 0.9, 0.999, 1e-8, step) == 0
        wr, mr, vr = co.adam(wr, g.astype(np.float64), mr, vr, 1e-2, 0.9, 0.999, 1e-8, step)
    got = Wt.cpu().numpy()
    assert np.abs(got - wr).max() <= 1e-6 * np.abs(wr).max()
    assert np.array_equal(Wb.cpu().numpy().view(np.uint16), co.bf16_bits(got))


def test_network_gradient_matches_oracle_chain():
    """Four layers (3 -> 8 -> 8 -> 8 -> 5, ReLU between) through the
    module's forward/backward against the oracle's chain rule."""
    import torch
    from nemo3d_b200 import warmstart as ws
    G, n = 5, 2
    net = ws.WarmStartNet(G=G, width=8, k=4, seed=1)
    rng = np.random.default_rng(5)
    x = rng.random((n, 3, G ** 3)).astype(np.float32)
    env = rng.random((n, 4, G ** 3)).astype(np.float32)
    sig = rng.normal(size=n).astype(np.float32)
    acts = net.forward(_t(x))
    _, dout, _ = net.loss(acts[-1], _t(env), _t(sig), 1.0)
    net.backward(acts, dout)
    # oracle chain on the same bf16 weights
    ws_ = [co.bf16_round(L["w"].cpu().numpy()) for L in net.layers]
    bs = [L["b"].cpu().numpy().astype(np.float64) for L in net.layers]
    a = [x.astype(np.float64).reshape(n, 3, G, G, G)]
    for i in range(4):
        a.append(co.conv3d_fwd(a[-1], ws_[i], bs[i], relu=i < 3))
    _, g, _ = co.loss(a[-1], env.astype(np.float64).reshape(n, 4, G, G, G), sig, 1.0)
    for i in range(3, -1, -1):
        dx, dw, db = co.conv3d_bwd(a[i], ws_[i], g)
        gw = net.layers[i]["gw"].cpu().numpy()
        gb = net.layers[i]["gb"].cpu().numpy()
        assert np.abs(gw - dw).max() <= 1e-4 * np.abs(dw).max(), i
        assert np.abs(gb - db).max() <= 1e-4 * max(np.abs(db).max(), 1e-12), i
        if i:
            g = dx * (a[i] > 0)


def test_features_and_start_vector_match_oracle():
    import torch
    from nemo3d_b200 import warmstart as ws
    from nemo3d_b200.tbgpu import Hamiltonian
    st = workloads.lens_dot((10, 9, 7), base_nm=3.0, height_nm=1.2, x_in=0.7, seed=2)
    H = Hamiltonian(st, "sp3d5s*_so", ws._mats())
    G = 6
    f = ws.features(H, G).cpu().numpy()
    ref = co.features(st.types, st.dsp, G, materials.SPECIES["In"])
    assert np.array_equal(f[:2], ref[:2].astype(np.float32))
    assert np.abs(f[2] - ref[2]).max() <= 1e-5 * np.abs(ref[2]).max()
    rng = np.random.default_rng(6)
    env = rng.random((8, G ** 3)).astype(np.float32)
    prof = rng.random((8, 2, H.nb)).astype(np.float32)
    u = workloads.random_start(H.n, seed=1)
    U, R = _t(u, torch.float64), torch.empty(2 * H.n, dtype=torch.float64, device="cuda")
    assert ws._lib().tbgpu_ws_start_vector(H._ctx, ws._ptr(_t(env)), ws._ptr(_t(prof)), 8, G,
                                          0.05, ws._ptr(U), ws._ptr(R)) == 0
    site = H.export_pattern()[0]
    uc = u[0::2] + 1j * u[1::2]
    want = co.start_vector(site, (st.nx, st.ny, st.nz), H.nb, env.astype(np.float64),
                           prof.astype(np.float64), G, 0.05, uc)
    r = R.cpu().numpy()
    got = r[0::2] + 1j * r[1::2]
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
    H.close()


def test_training_lowers_the_loss():
    import torch
    from nemo3d_b200 import warmstart as ws
    G, n = 8, 6
    net = ws.WarmStartNet(G=G, seed=0)
    rng = np.random.default_rng(7)
    x = _t(rng.random((n, 3, G ** 3)))
    env = _t(np.repeat(x[:, :1].cpu().numpy(), 8, axis=1) * 2.0)  # envelopes = 2 x In fraction
    sig = _t(x[:, 0].mean(1).cpu().numpy() * 3.0)
    first = net.train_step(x, env, sig, lr=3e-3)
    for _ in range(150):
        last = net.train_step(x, env, sig, lr=3e-3)
    assert last < 0.1 * first


def test_warm_solve_finds_the_cold_levels():
    from nemo3d_b200 import warmstart as ws
    from nemo3d_b200.tbgpu import Hamiltonian
    G = 8
    train = [ws.solve_sample(workloads.random_lens(s, cells=(16, 16, 12)), G) for s in range(3)]
    train = [t for t in train if t is not None]
    assert len(train) >= 2
    net = ws.WarmStartNet(G=G, seed=0)
    net.fit(train, epochs=20, batch=2)
    st = workloads.random_lens(100, cells=(16, 16, 12))
    H = Hamiltonian(st, ws.MODEL, ws._mats())
    cold = ws.warm_solve(H, None)
    warm = ws.warm_solve(H, net)
    assert not cold["warm"]
    assert cold["edges"] is not None and warm["edges"] is not None
    assert np.abs(warm["edges"] - cold["edges"]).max() < 1e-6
    H.close()
