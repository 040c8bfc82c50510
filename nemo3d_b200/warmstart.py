"""Learned warm start of the Lanczos solve.

A 3-D convolutional network (4 layers, 32 channels, 3x3x3 kernels, bf16
weights with float accumulation) reads per-voxel features of a structure on
a G^3 grid over its cells (In fraction, occupancy, displacement length) and
predicts the in-gap shift sigma (grid mean of its last channel) and K = 8
band-edge envelopes (4 hole and 4 electron levels; sqrt of each state's
probability per voxel).  The envelopes, with orbital profiles averaged over
the training solves, shape the Lanczos start vector: the uniform random
start of the plain method times sqrt(sum_k env_k^2 prof_k + floor) per atom
and orbital.  sigma places the two search windows.  The plain cold start
stays the fallback: a warm solve that finds fewer states than requested is
repeated cold.

Training data come from plain solves of randomized dots
(``workloads.random_lens``); forward, backward, loss and Adam run in the
project's CUDA kernels (``csrc/warmstart.cu``) on device buffers held by
torch.  No counterpart in the reference (its start vector is rand() or a
file, eigen/src/lanczos.c:1823-1900).
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import materials, tbgpu, workloads

K = 8             # envelopes: 4 hole levels, 4 electron levels (ascending)
IN_CH = 3
SIGMA0, SIGMA_SCALE = 1.2, 0.1   # sigma is learned as (sigma - SIGMA0) / SIGMA_SCALE
WINDOW = 1.1      # width of each search window beside sigma (eV)
MAXVEC = 12       # eigenvector slots of a training solve (the solver may return
                  # one level more than requested per window)
MODEL = "sp3d5s*_so"


def _mats():
    return [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]


def _lib():
    L = tbgpu._lib()
    if not getattr(L, "_ws_bound", False):
        vp, ip, fp, lp = C.c_void_p, C.c_int, C.c_float, C.c_long
        L.tbgpu_ws_features.argtypes = [vp, ip, ip, vp]
        L.tbgpu_ws_conv3d_fwd.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, ip]
        L.tbgpu_ws_conv3d_bwd_data.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip]
        L.tbgpu_ws_conv3d_bwd_weight.argtypes = [vp, vp, vp, vp, vp, ip, ip, ip, ip]
        L.tbgpu_ws_loss.argtypes = [vp, vp, vp, ip, ip, ip, fp, vp, vp, vp]
        L.tbgpu_ws_adam.argtypes = [vp, vp, vp, vp, vp, lp, fp, fp, fp, fp, ip]
        L.tbgpu_ws_start_vector.argtypes = [vp, vp, vp, ip, ip, fp, vp, vp]
        L._ws_bound = True
    return L


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check(rc, name):
    if rc:
        raise tbgpu.TbgpuError(rc, name)


def _bf16(w):
    import torch
    return w.to(torch.bfloat16).view(torch.int16).contiguous()


def features(H, G: int):
    """[3, G^3] float32 device tensor of the structure behind Hamiltonian H."""
    import torch
    f = torch.empty((IN_CH, G ** 3), dtype=torch.float32, device="cuda")
    _check(_lib().tbgpu_ws_features(H._ctx, G, materials.SPECIES["In"], _ptr(f)),
           "tbgpu_ws_features")
    return f


class WarmStartNet:
    """The network, its Adam state and the orbital profiles."""

    def __init__(self, G: int = 16, width: int = 32, k: int = K, seed: int = 0):
        import torch
        self.G, self.k, self.width = G, k, width
        chans = [IN_CH, width, width, width, k + 1]
        gen = torch.Generator().manual_seed(seed)
        self.layers = []
        for cin, cout in zip(chans[:-1], chans[1:]):
            std = (2.0 / (cin * 27)) ** 0.5
            w = (torch.randn(cout, cin, 27, generator=gen) * std).float().cuda()
            b = torch.zeros(cout, device="cuda")
            self.layers.append(dict(
                cin=cin, cout=cout, w=w, b=b, wbf=_bf16(w),
                bbf=torch.empty(cout, dtype=torch.int16, device="cuda"),
                mw=torch.zeros_like(w), vw=torch.zeros_like(w),
                mb=torch.zeros_like(b), vb=torch.zeros_like(b),
                gw=torch.zeros_like(w), gb=torch.zeros_like(b)))
        self.step = 0
        self.prof = None  # [k, 2, nb] orbital profiles (numpy), set by fit()

    # -- kernels ---------------------------------------------------------
    def forward(self, x):
        """x [n, 3, G^3] float32 -> activations of every layer (input first)."""
        import torch
        n, G = x.shape[0], self.G
        acts = [x.contiguous()]
        for li, L in enumerate(self.layers):
            out = torch.empty((n, L["cout"], G ** 3), dtype=torch.float32, device="cuda")
            relu = int(li < len(self.layers) - 1)
            _check(_lib().tbgpu_ws_conv3d_fwd(_ptr(acts[-1]), _ptr(L["wbf"]), _ptr(L["b"]),
                                              _ptr(out), n, L["cin"], L["cout"], G, relu),
                   "tbgpu_ws_conv3d_fwd")
            acts.append(out)
        return acts

    def backward(self, acts, dout):
        """Fill every layer's gw, gb from dout = dL/d(last output)."""
        import torch
        n, G = dout.shape[0], self.G
        g = dout
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            act = acts[li + 1] if li < len(self.layers) - 1 else None
            _check(_lib().tbgpu_ws_conv3d_bwd_weight(_ptr(acts[li]), _ptr(g), _ptr(act),
                                                     _ptr(L["gw"]), _ptr(L["gb"]), n, L["cin"],
                                                     L["cout"], G),
                   "tbgpu_ws_conv3d_bwd_weight")
            if li > 0:
                din = torch.empty_like(acts[li])
                _check(_lib().tbgpu_ws_conv3d_bwd_data(_ptr(g), _ptr(act), _ptr(L["wbf"]),
                                                       _ptr(din), n, L["cin"], L["cout"], G),
                       "tbgpu_ws_conv3d_bwd_data")
                g = din

    def loss(self, out, env, sigma, w_sigma=1.0):
        """(loss tensor [1], dout, sigma_pred) for targets env [n, k, G^3],
        sigma [n] (normalised)."""
        import torch
        n = out.shape[0]
        dout = torch.empty_like(out)
        sp = torch.empty(n, dtype=torch.float32, device="cuda")
        ls = torch.empty(1, dtype=torch.float32, device="cuda")
        _check(_lib().tbgpu_ws_loss(_ptr(out), _ptr(env), _ptr(sigma), n, self.k, self.G,
                                    float(w_sigma), _ptr(dout), _ptr(sp), _ptr(ls)),
               "tbgpu_ws_loss")
        return ls, dout, sp

    def adam(self, lr=2e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        for L in self.layers:
            _check(_lib().tbgpu_ws_adam(_ptr(L["w"]), _ptr(L["wbf"]), _ptr(L["gw"]), _ptr(L["mw"]),
                                        _ptr(L["vw"]), L["w"].numel(), lr, b1, b2, eps,
                                        self.step), "tbgpu_ws_adam")
            _check(_lib().tbgpu_ws_adam(_ptr(L["b"]), _ptr(L["bbf"]), _ptr(L["gb"]), _ptr(L["mb"]),
                                        _ptr(L["vb"]), L["b"].numel(), lr, b1, b2, eps,
                                        self.step), "tbgpu_ws_adam")

    def train_step(self, x, env, sigma, lr=2e-3, w_sigma=1.0) -> float:
        acts = self.forward(x)
        ls, dout, _ = self.loss(acts[-1], env, sigma, w_sigma)
        self.backward(acts, dout)
        self.adam(lr)
        return float(ls.item())

    def predict(self, x):
        """x [n, 3, G^3] -> (env [n, k, G^3] tensor, sigma [n] numpy, eV)."""
        import torch
        out = self.forward(x)[-1]
        sp = torch.empty(out.shape[0], dtype=torch.float32, device="cuda")
        _check(_lib().tbgpu_ws_loss(_ptr(out), None, None, out.shape[0], self.k, self.G, 0.0,
                                    None, _ptr(sp), None), "tbgpu_ws_loss")
        return out[:, :self.k].contiguous(), SIGMA0 + SIGMA_SCALE * sp.cpu().numpy().astype(
            np.float64)

    # -- data and training ----------------------------------------------
    def fit(self, samples, epochs=300, batch=8, lr=2e-3, w_sigma=1.0, seed=0):
        """Train on samples from ``solve_sample`` (features, env, sigma, prof);
        returns the loss per epoch."""
        import torch
        X = torch.stack([s["features"] for s in samples])
        E = torch.stack([torch.from_numpy(s["env"]).float() for s in samples]).cuda()
        S = torch.tensor([(s["sigma"] - SIGMA0) / SIGMA_SCALE for s in samples],
                         dtype=torch.float32, device="cuda")
        self.prof = np.mean([s["prof"] for s in samples], axis=0)
        rng = np.random.default_rng(seed)
        hist = []
        for _ in range(epochs):
            order = rng.permutation(len(samples))
            tot = 0.0
            for b0 in range(0, len(order), batch):
                idx = torch.from_numpy(order[b0:b0 + batch]).cuda()
                tot += self.train_step(X[idx], E[idx], S[idx], lr, w_sigma) * len(idx)
            hist.append(tot / len(samples))
        return hist


def env_scale(G: int) -> float:
    """Target scale: a state spread over G^3/64 voxels gets envelopes of
    about 1."""
    return float(np.sqrt(G ** 3 / 64.0))


def targets(H, values, vectors, G: int):
    """Envelopes [k, G^3], sigma (eV) and orbital profiles [k, 2, nb] of a
    solved structure (values ascending, 4 hole then 4 electron levels,
    vectors [k, dimension] complex)."""
    site = H.export_pattern()[0].astype(np.int64)
    nb = H.nb
    st = H.structure
    nx, ny, nz = st.nx, st.ny, st.nz
    cell = site >> 3
    kc = cell % nz
    jc = (cell // nz) % ny
    ic = cell // (nz * ny)
    vox = ((ic * G) // nx * G + (jc * G) // ny) * G + (kc * G) // nz
    sub = ((site & 7) >= 4).astype(np.int64)
    k = vectors.shape[0]
    env = np.zeros((k, G ** 3))
    prof = np.zeros((k, 2, nb))
    norb = nb // 2 if nb in (10, 20) else nb
    for q in range(k):
        p = np.abs(vectors[q].reshape(-1, nb)) ** 2
        p /= p.sum()
        env[q] = np.sqrt(np.bincount(vox, p.sum(1), G ** 3)) * env_scale(G)
        for s in (0, 1):
            w = p[sub == s].sum(0)
            if nb == 2 * norb:  # spin-summed orbital weight, both spins alike
                w = np.tile(w[:norb] + w[norb:], 2) / 2
            prof[q, s] = w
    return env, 0.5 * (values[3] + values[4]), prof


def solve_kw(sigma: float):
    """The search windows beside sigma: 4 hole levels below, 4 electron
    levels above."""
    return dict(requested1=4, requested2=4, emin1=sigma - WINDOW, emax1=sigma,
                emin2=sigma, emax2=sigma + WINDOW, tolerance=1e-7, imax=20000)


def band_edges(values, sigma: float):
    """Indices of the 4 highest levels below sigma and the 4 lowest above
    (ascending), or None when either side has fewer than 4."""
    v = np.asarray(values)
    lo = np.nonzero(v <= sigma)[0]
    hi = np.nonzero(v > sigma)[0]
    if lo.size < 4 or hi.size < 4:
        return None
    return np.concatenate([lo[-4:], hi[:4]])


def solve_sample(st, G: int, seed: int = 0):
    """Plain cold solve of one structure; returns the training sample and
    the solve's iteration count and wall time."""
    H = tbgpu.Hamiltonian(st, MODEL, _mats())
    try:
        r0 = workloads.random_start(H.n, seed=seed)
        t0 = time.perf_counter()
        res = H.eigensolve_lanczos(r0, vectors=MAXVEC, **solve_kw(SIGMA0))
        wall = time.perf_counter() - t0
        idx = band_edges(res["values"], SIGMA0)
        if idx is None or idx[-1] >= MAXVEC:
            return None
        env, sigma, prof = targets(H, np.asarray(res["values"])[idx], res["vectors"][idx], G)
        return dict(features=features(H, G), env=env.astype(np.float32), sigma=sigma, prof=prof,
                    values=res["values"], iterations=res["iterations"], wall=wall)
    finally:
        H.close()


def warm_start_vector(H, net: WarmStartNet, seed: int = 0, floor_frac: float = 0.02):
    """(r0 host vector, predicted sigma) for Hamiltonian H."""
    import torch
    G = net.G
    env, sig = net.predict(features(H, G)[None])
    env = env[0].clamp(min=0.0).contiguous()
    prof = torch.from_numpy(net.prof.astype(np.float32)).cuda().contiguous()
    u = torch.from_numpy(workloads.random_start(H.n, seed=seed)).cuda()
    r0 = torch.empty_like(u)
    peak = float((env ** 2).sum(0).max().item()) * float(net.prof.max())
    floor_w = max(floor_frac * peak, 1e-12)
    _check(_lib().tbgpu_ws_start_vector(H._ctx, _ptr(env), _ptr(prof), net.k, G, floor_w, _ptr(u),
                                        _ptr(r0)), "tbgpu_ws_start_vector")
    return r0.cpu().numpy(), float(sig[0])


def warm_solve(H, net: WarmStartNet | None, seed: int = 0, vectors: int = 0):
    """Solve with the learned start and windows beside the predicted sigma;
    falls back to the plain cold start (sigma = SIGMA0) when there is no
    network or the warm solve finds fewer than 4 levels on either side.
    Returns the solver's result dict plus 'warm' (bool), 'sigma' and 'edges'
    (the 4 + 4 band-edge levels, ascending, or None)."""
    if net is not None:
        r0, sig = warm_start_vector(H, net, seed)
        res = H.eigensolve_lanczos(r0, vectors=vectors, **solve_kw(sig))
        idx = band_edges(res["values"], sig)
        if idx is not None:
            res.update(warm=True, sigma=sig, edges=np.asarray(res["values"])[idx])
            return res
    r0 = workloads.random_start(H.n, seed=seed)
    res = H.eigensolve_lanczos(r0, vectors=vectors, **solve_kw(SIGMA0))
    idx = band_edges(res["values"], SIGMA0)
    res.update(warm=False, sigma=SIGMA0,
               edges=None if idx is None else np.asarray(res["values"])[idx])
    return res
