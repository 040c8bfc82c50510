"""CPU restatement of the warm-start network kernels (nemo3d_b200/csrc/warmstart.cu).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
kernels.  The product never imports it.

Plain numpy in float64 on bf16-rounded weights: 3x3x3 convolution with zero
padding (tap t = (dx+1)*9 + (dy+1)*3 + dz+1, voxel (x*G + y)*G + z), its
gradients with respect to input, weights and bias, the envelope/sigma loss,
an Adam step, the structure features and the start-vector map.  The warm
start has no counterpart in the reference; these restate the definitions in
the kernel file's header, not reference code.
"""

from __future__ import annotations

import numpy as np

OFFS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def bf16_round(w: np.ndarray) -> np.ndarray:
    """float32 -> bf16 (round to nearest even) -> float64."""
    u = np.asarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(w: np.ndarray) -> np.ndarray:
    u = np.asarray(w, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def _shift(a: np.ndarray, d) -> np.ndarray:
    """b[..., x, y, z] = a[..., x + dx, y + dy, z + dz], zero outside."""
    out = np.zeros_like(a)
    G = a.shape[-1]
    src = [slice(max(0, o), G + min(0, o)) for o in d]
    dst = [slice(max(0, -o), G + min(0, -o)) for o in d]
    out[(...,) + tuple(dst)] = a[(...,) + tuple(src)]
    return out


def conv3d_fwd(x, w, b, relu=False):
    """x [n][cin][G][G][G], w [cout][cin][27] (float64), b [cout]."""
    out = np.zeros((x.shape[0], w.shape[0]) + x.shape[2:])
    for t, d in enumerate(OFFS):
        out += np.einsum("oc,ncxyz->noxyz", w[:, :, t], _shift(x, d))
    out += b[None, :, None, None, None]
    return np.maximum(out, 0.0) if relu else out


def conv3d_bwd(x, w, g):
    """Gradients of sum(g * conv3d_fwd(x, w, b)) (g already masked by the
    ReLU): returns (dx, dw, db)."""
    dx = np.zeros_like(x)
    dw = np.zeros_like(w)
    for t, d in enumerate(OFFS):
        xs = _shift(x, d)
        dw[:, :, t] = np.einsum("noxyz,ncxyz->oc", g, xs)
        dx += _shift(np.einsum("oc,noxyz->ncxyz", w[:, :, t], g), tuple(-o for o in d))
    db = g.sum(axis=(0, 2, 3, 4))
    return dx, dw, db


def loss(out, env, sigma, w_sigma):
    """out [n][k+1][G^3...]: (loss, dout, sigma_pred)."""
    n, k1 = out.shape[:2]
    k = k1 - 1
    G3 = out[0, 0].size
    sp = out[:, k].reshape(n, -1).mean(axis=1)
    d = np.zeros_like(out)
    diff = out[:, :k] - env
    L = (diff ** 2).sum() / (n * k * G3) + w_sigma * ((sp - sigma) ** 2).mean()
    d[:, :k] = 2 * diff / (n * k * G3)
    d[:, k] = (2 * w_sigma * (sp - sigma) / n / G3)[:, None, None, None]
    return L, d, sp


def adam(w, g, m, v, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    lr_t = lr * np.sqrt(1 - b2 ** step) / (1 - b1 ** step)
    return w - lr_t * m / (np.sqrt(v) + eps), m, v


def voxel_of(i, n, G):
    return (np.asarray(i, np.int64) * G) // n


def features(types, dsp, G, in_species):
    """types [nx][ny][nz][8], dsp [nx][ny][nz][8][3] nm or None -> [3][G^3]."""
    nx, ny, nz = types.shape[:3]
    vx, vy, vz = voxel_of(np.arange(nx), nx, G), voxel_of(np.arange(ny), ny, G), \
        voxel_of(np.arange(nz), nz, G)
    vid = (vx[:, None, None] * G + vy[None, :, None]) * G + vz[None, None, :]
    G3 = G ** 3
    occ = types > 0
    cat = occ[..., :4]
    nin = (types[..., :4] == in_species).sum(-1)
    f = np.zeros((3, G3))
    ncat = np.bincount(vid.ravel(), cat.sum(-1).ravel(), G3)
    nsite = np.bincount(vid.ravel(), np.full(vid.size, 8.0), G3)
    nocc = np.bincount(vid.ravel(), occ.sum(-1).ravel(), G3)
    f[0] = np.divide(np.bincount(vid.ravel(), nin.ravel(), G3), ncat,
                     out=np.zeros(G3), where=ncat > 0)
    f[1] = np.divide(nocc, nsite, out=np.zeros(G3), where=nsite > 0)
    if dsp is not None:
        ln = np.where(occ, np.linalg.norm(dsp, axis=-1), 0.0).sum(-1)
        f[2] = np.divide(np.bincount(vid.ravel(), ln.ravel(), G3) * 1000.0, nocc,
                         out=np.zeros(G3), where=nocc > 0)
    return f


def start_vector(atom_site, dims, nb, env, prof, G, floor_w, u):
    """atom_site [natoms] site indices, env [k][G^3], prof [k][2][nb], u
    complex [natoms * nb] -> r0 complex."""
    nx, ny, nz = dims
    s = np.asarray(atom_site, np.int64)
    m = s & 7
    cell = s >> 3
    k = cell % nz
    j = (cell // nz) % ny
    i = cell // (nz * ny)
    v = (voxel_of(i, nx, G) * G + voxel_of(j, ny, G)) * G + voxel_of(k, nz, G)
    sub = (m >= 4).astype(np.int64)
    w2 = np.full((s.size, nb), floor_w)
    for q in range(env.shape[0]):
        w2 += (env[q][v] ** 2)[:, None] * prof[q][sub]
    return (u.reshape(-1, nb) * np.sqrt(w2)).ravel()
