"""Oracle for the learned level selector (TEST INFRASTRUCTURE): a numpy
restatement, in FP64, of the selector's per-panel descriptor, its 8 pair
features and the MLP's mean cross-entropy with its gradient.

The selector has no counterpart in the reference, so nothing of the reference
pins it: its labels are the plain ball-test walk's levels, which the GPU
parity tests already pin against the oracle's restatement of
lap3dsdlpmat_levels_r64 (patch_refine_mod.f90:516-551).  The gradient here is
checked against finite differences (tests/test_oracle.py), the GPU's features
and gradient against this file (tests/test_gpu_selector.py).

Only tests/ may import this module.
"""
import numpy as np

F, H, NC = 8, 64, 5
OW1, OB1, OW2, OB2, OW3, OB3 = 0, 512, 576, 4672, 4736, 5056
NW = OB3 + NC


def panel_descriptor(sx, snx, sw):
    """(c, nb, e1, e2, D, kappa, ln aspect) of one panel: nodes sx (hd, 3),
    normals snx (hd, 3), weights sw (hd,)"""
    s0 = sw.sum()
    c = (sw[:, None] * sx).sum(0) / s0
    nb = (sw[:, None] * snx).sum(0)
    nb = nb / np.linalg.norm(nb)
    a = sx[0] - c
    a = a - (a @ nb) * nb
    e1 = a / np.linalg.norm(a)
    e2 = np.cross(nb, e1)
    kap = np.linalg.norm(snx - nb, axis=1).max()
    y = sx - c
    u, v = y @ e1, y @ e2
    ixx, iyy, ixy = (sw * u * u).sum(), (sw * v * v).sum(), (sw * u * v).sum()
    tr = 0.5 * (ixx + iyy)
    dt = np.sqrt(0.25 * (ixx - iyy) ** 2 + ixy ** 2)
    l1, l2 = tr + dt, max(tr - dt, 1e-300)
    return c, nb, e1, e2, np.sqrt(s0), kap, 0.5 * np.log(l1 / l2)


def features(x, desc, sx):
    """the 8 features of targets x (m, 3) against one panel"""
    c, nb, e1, e2, D, kap, lna = desc
    d = x - c
    r = np.linalg.norm(d, axis=1)
    lg = lambda v: np.log10(np.maximum(v, 1e-12))
    h = d @ nb
    mind = np.sqrt(((x[:, None, :] - sx[None, :, :]) ** 2).sum(-1).min(1))
    f = np.empty((x.shape[0], F))
    f[:, 0] = lg(r / D)
    f[:, 1] = np.tanh((d @ e1) / D)
    f[:, 2] = np.tanh((d @ e2) / D)
    f[:, 3] = np.where(r > 0, h / np.where(r > 0, r, 1.0), 0.0)
    f[:, 4] = lg(np.abs(h) / D)
    f[:, 5] = kap
    f[:, 6] = lna
    f[:, 7] = lg(mind / D)
    return f


def pair_features(npan, hd, sx, snx, sw, tcx, tcxi):
    """features of every near pair, panel by panel (CSR tcxi, one-based)"""
    sx, snx = sx.reshape(-1, 3), snx.reshape(-1, 3)
    tcx = tcx.reshape(-1, 3)
    out = np.empty((tcx.shape[0], F))
    for p in range(npan):
        sl = slice(p * hd, (p + 1) * hd)
        a, b = tcxi[p] - 1, tcxi[p + 1] - 1
        if b > a:
            out[a:b] = features(tcx[a:b], panel_descriptor(sx[sl], snx[sl], sw[sl]), sx[sl])
    return out


def bf16(a):
    """float32 values rounded to BF16 (nearest, ties to even), as float64"""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[OW1:OB1].reshape(F, H), w[OB1:OW2], w[OW2:OB2].reshape(H, H), w[OB2:OW3],
            w[OW3:OB3].reshape(H, NC), w[OB3:NW])


def loss_grad(w, x, y, bf=False):
    """mean cross-entropy of the MLP (ReLU, ReLU, softmax) and its gradient;
    bf: the library's BF16 operands (weights, inputs and hidden activations
    rounded to BF16, sums exact), the gradient taken with respect to the
    rounded weights"""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(r(w) if bf else w)
    x = r(x)
    a1 = x @ W1 + b1
    h1 = r(np.maximum(a1, 0.0))
    a2 = h1 @ W2 + b2
    h2 = r(np.maximum(a2, 0.0))
    z = h2 @ W3 + b3
    zm = z.max(1, keepdims=True)
    e = np.exp(z - zm)
    p = e / e.sum(1, keepdims=True)
    n = x.shape[0]
    loss = float((np.log(e.sum(1)) + zm[:, 0] - z[np.arange(n), y]).mean())
    dz = p.copy()
    dz[np.arange(n), y] -= 1.0
    dz /= n
    dh2 = (dz @ W3.T) * (a2 > 0)
    dh1 = (dh2 @ W2.T) * (a1 > 0)
    g = np.concatenate([(x.T @ dh1).ravel(), dh1.sum(0), (h1.T @ dh2).ravel(), dh2.sum(0), (h2.T @ dz).ravel(),
                        dz.sum(0)])
    return loss, g


def predict(w, x):
    """class and softmax probability of each row of x"""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.maximum(np.asarray(x, dtype=np.float64) @ W1 + b1, 0.0)
    z = np.maximum(h1 @ W2 + b2, 0.0) @ W3 + b3
    e = np.exp(z - z.max(1, keepdims=True))
    p = e / e.sum(1, keepdims=True)
    return p.argmax(1), p.max(1)
