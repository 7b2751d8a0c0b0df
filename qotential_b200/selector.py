"""Training data and training for the learned level selector (no reference
counterpart): seeded surfaces of the batched family, their near pairs
(on-surface nodes plus off-surface points at seeded normal offsets), each
pair's 8 features and a label, and Adam on the GPU (qol_selector_train).

Two label sets.  "walk": the level the plain ball-test walk gives the pair,
so a selector trained on them reproduces the walk where it is confident (the
library's mode 1).  "error": the lowest level whose row is within a
tolerance of the finest level's (error_levels: every direct pair computed on
each level by qol_selector_force_level), capped at the walk's level, RRQ for
the pairs the walk sends to RRQ; the library's mode 2 uses a prediction below
the walk's level after its two-level check."""
import numpy as np

from . import geometry as G
from . import qol_getnearquad_lap_rrq_dev, qol_selector_features, qol_selector_force_level, qol_selector_train


def error_levels(npan, nterms, P, tcx, tcxrow, tcxi, walk_level, distff=1.4):
    """(ntcx, 4) row errors of levels 1..4 against level 4 per near pair:
    max(1-norm of the single-layer row difference / D, 1-norm of the
    double-layer row difference), D = sqrt(panel area) (the check's scale);
    zero for RRQ pairs (walk level 5).  Computed on the GPU from four
    getnearquad runs with every direct pair forced onto one level."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    hd = nterms * (nterms + 1) // 2
    nq = nterms + 2
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
    D = {k: t(P[k]) for k in ("sx", "snx", "sw", "rts", "rps")}
    xi = np.asarray(tcxi, np.int64)
    ntcx = int(xi[-1] - 1)
    tx, row, xid = t(tcx), t(tcxrow, torch.int64), t(xi, torch.int64)
    nnz = ntcx * hd
    out = (torch.empty(nnz, dtype=torch.int64, device=dev), torch.empty(nnz, dtype=torch.int64, device=dev),
           torch.empty(nnz, dtype=torch.float64, device=dev), torch.empty(nnz, dtype=torch.float64, device=dev))
    m = torch.as_tensor(np.diff(xi), device=dev)
    pan = torch.repeat_interleave(torch.arange(npan, device=dev), hd * m)      # panel of each COO entry
    local = torch.arange(nnz, device=dev) - (xid[:-1] - 1)[pan] * hd
    pair = (xid[:-1] - 1)[pan] + local % m[pan]                               # block column-major order
    diam = torch.sqrt(D["sw"].reshape(npan, hd).sum(1))[pan]
    err = torch.zeros((ntcx, 4), dtype=torch.float64, device=dev)

    def run(level):
        qol_selector_force_level(level)
        qol_getnearquad_lap_rrq_dev(npan, nterms, nq, D["sx"], D["snx"], D["sw"], D["rts"], D["rps"], tx, row, xid,
                                    nq, distff, 30, out, stream=torch.cuda.current_stream().cuda_stream)

    try:
        run(4)
        vs4, vd4 = out[2].clone(), out[3].clone()
        for lv in (1, 2, 3):
            run(lv)
            es = torch.zeros(ntcx, dtype=torch.float64, device=dev).index_add_(0, pair, (out[2] - vs4).abs() / diam)
            ed = torch.zeros(ntcx, dtype=torch.float64, device=dev).index_add_(0, pair, (out[3] - vd4).abs())
            err[:, lv - 1] = torch.maximum(es, ed)
    finally:
        qol_selector_force_level(0)
    e = err.cpu().numpy()
    e[np.asarray(walk_level) > 4] = 0.0
    return e


def error_labels(err, walk_level, tol):
    """classes 0..4: the lowest level (0-based) whose row error is <= tol,
    capped at the walk's level (the library lowers the walk's level, never
    raises it); 4 (RRQ) where the walk gives RRQ"""
    ok = np.asarray(err) <= tol
    walk = np.asarray(walk_level).astype(np.int64)
    low = np.minimum(np.where(ok.any(1), ok.argmax(1), 3), walk - 1)
    return np.where(walk > 4, 4, low).astype(np.int8)


def training_set(n_pairs=1_000_000, seed=11, orders=(4, 6, 8, 10, 12), noff=5000, max_grid=(8, 32), labels="walk",
                 tol=1e-8):
    """(features (n, 8) float32, classes (n,) int8, surfaces used) from seeded
    family surfaces until at least n_pairs pairs are collected; labels "walk"
    or "error" (at tolerance tol)"""
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
        if labels == "error":
            labs.append(error_labels(error_levels(npan, nterms, P, tcx, tcxrow, tcxi, lev), lev, tol))
        else:
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
