"""Training data and training for the learned level selector (no reference
counterpart): seeded surfaces of the batched family, their near pairs
(on-surface nodes plus off-surface points at seeded normal offsets), each
pair's 8 features and the level the plain ball-test walk gives it, and Adam
on the GPU (qol_selector_train).  The labels are the plain walk's own
decisions, so a selector trained here reproduces the plain walk where it is
confident; the library accepts a prediction only after the ball check at the
predicted level."""
import numpy as np

from . import geometry as G
from . import qol_selector_features, qol_selector_train


def training_set(n_pairs=1_000_000, seed=11, orders=(4, 6, 8, 10, 12), noff=5000, max_grid=(8, 32)):
    """(features (n, 8) float32, classes (n,) int8, surfaces used) from seeded
    family surfaces until at least n_pairs pairs are collected"""
    rng = np.random.default_rng(seed)
    feats, labs, used = [], [], 0
    total = 0
    while total < n_pairs:
        surf = G.family_surface(rng)
        k = int(rng.choice(orders))
        nterms = k + 1
        mp = int(rng.integers(4, max_grid[0] + 1))
        np_ = int(rng.integers(2 * mp, max_grid[1] + 1))
        P = G.panels(surf, mp, np_, nterms, split=False)
        hd = nterms * (nterms + 1) // 2
        T = np.concatenate([P["sx"], G.off_surface_targets(P, noff, int(rng.integers(1 << 30)), hd)])
        tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
        npan = P["sw"].size // hd
        f, lev = qol_selector_features(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                       tcxrow, tcxi, nterms + 2)
        feats.append(f)
        labs.append((lev - 1).astype(np.int8))
        total += f.shape[0]
        used += 1
    return np.concatenate(feats), np.concatenate(labs), used


def predict(w, feat):
    """class and softmax probability of each feature row with weights w (FP32
    masters; weights, features and activations rounded to BF16 as the library's
    kernels use them)"""
    w = np.asarray(w, dtype=np.float32)
    u = w.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    wb = u.view(np.float32).astype(np.float64)
    W1, b1 = wb[0:512].reshape(8, 64), wb[512:576]
    W2, b2 = wb[576:4672].reshape(64, 64), wb[4672:4736]
    W3, b3 = wb[4736:5056].reshape(64, 5), wb[5056:5061]

    def r(a):  # BF16 operands, as the library's kernels
        v = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
        v = ((v + 0x7FFF + ((v >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
        return v.view(np.float32).astype(np.float64)

    h = r(np.maximum(r(feat) @ W1 + b1, 0.0))
    z = r(np.maximum(h @ W2 + b2, 0.0)) @ W3 + b3
    e = np.exp(z - z.max(1, keepdims=True))
    p = e / e.sum(1, keepdims=True)
    return p.argmax(1), p.max(1)


def train(n_pairs=1_000_000, seed=11, epochs=20, batch=16384, lr=3e-3):
    """(weights, per-epoch loss, training accuracy, pairs, surfaces) on a fresh
    training set"""
    feat, lab, used = training_set(n_pairs, seed)
    w, loss = qol_selector_train(feat, lab, epochs=epochs, batch=batch, lr=lr, seed=seed)
    cls, _ = predict(w, feat)
    return w, loss, float((cls == lab).mean()), int(lab.size), used
