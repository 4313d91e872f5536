"""CPU double-precision oracle of the learned proposal network (test infrastructure only).

The proposal network has no counterpart in the reference; this module restates, in numpy float64,
what the library's kernels compute, so the tests can check them:

  * features and label bytes of a patch (k_prop_samples), from the descriptor and the table's
    partition -- the bin lookup is the reference's PatchPartition1D::get_bin
    (patchtable/patchtable.h:1298-1325) in float32 arithmetic;
  * the forward pass, the masked per-dimension softmax cross-entropy and its gradient, either in
    exact float64 or with BF16 rounding at the points where the GPU rounds (weights, inputs, the
    ReLU outputs and the back-propagated gradients), accumulation always in float64;
  * the exact top-8 cells of the factorised distribution, by enumeration.

Only tests import this module.
"""
from __future__ import annotations

import itertools

import numpy as np

IN, HIDDEN, OUT, DIMS, CLASSES, TOPK = 16, 128, 32, 6, 5, 8
NMAP = 16384


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even) through float32, returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out


def bf16_bits(x) -> np.ndarray:
    """Raw BF16 bit patterns (uint16) of bf16(x)."""
    return (np.ascontiguousarray(bf16(x), np.float32).view(np.uint32) >> 16).astype(np.uint16)


def unpack(vec: np.ndarray) -> dict:
    v = np.asarray(vec, np.float64)
    o, out = 0, {}
    for name, shp in (("W1", (HIDDEN, IN)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
                      ("W3", (OUT, HIDDEN)), ("b3", (OUT,))):
        n = int(np.prod(shp))
        out[name] = v[o:o + n].reshape(shp)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3")])


def get_bin(v, min_val, rng, to_bin) -> np.ndarray:
    """PatchPartition1D::get_bin in float32: idx = (v - min) * (NMAP - 1) / range, truncated and clamped."""
    v = np.asarray(v, np.float32)
    t = ((v - np.float32(min_val)) * np.float32(NMAP - 1)) / np.float32(rng)
    with np.errstate(invalid="ignore"):
        ok = (t >= np.float32(-2147483648.0)) & (t < np.float32(2147483648.0))
        idx = np.where(ok, np.trunc(np.where(ok, t, 0)), -2147483648).astype(np.int64)
    idx = np.clip(idx, 0, NMAP - 1)
    return np.asarray(to_bin)[idx]


def features(desc: np.ndarray, parts: list) -> tuple:
    """(features [P x 16] float32 before BF16 rounding, bins [P x G]) of descriptors desc [P x >=G].

    parts[d] = dict(centers, lsizes, rsizes, to_bin, min, range) of grid dimension d."""
    P = desc.shape[0]
    G = len(parts)
    f = np.zeros((P, IN), np.float32)
    bins = np.zeros((P, G), np.int64)
    for d, pa in enumerate(parts):
        x = desc[:, d].astype(np.float32)
        b = get_bin(x, pa["min"], pa["range"], pa["to_bin"])
        bins[:, d] = b
        c = np.asarray(pa["centers"], np.float32)[b]
        s = np.where(x >= c, np.asarray(pa["rsizes"], np.float32)[b], np.asarray(pa["lsizes"], np.float32)[b])
        with np.errstate(divide="ignore", invalid="ignore"):
            u = np.where(s > 0, (x - c) / np.where(s > 0, s, np.float32(1)), np.float32(0)).astype(np.float32)
            r = ((x - np.float32(pa["min"])) / np.float32(pa["range"])).astype(np.float32) if pa["range"] > 0 \
                else np.full(P, 0.5, np.float32)
        f[:, DIMS + d] = np.clip(u, -2, 2)
        f[:, d] = np.clip(r, -0.5, 1.5).astype(np.float32) - np.float32(0.5)
    return f, bins


def labels(bins_a: np.ndarray, bins_b: np.ndarray, nslices, valid: np.ndarray) -> np.ndarray:
    """Label bytes [P x 8] (see k_prop_samples) from the query and match bins."""
    P, G = bins_a.shape
    out = np.full((P, 8), 0xFF, np.uint8)
    off = bins_b - bins_a
    exact = valid & np.all((off >= -2) & (off <= 2), axis=1)
    for d in range(G):
        o = np.clip(off[:, d], -2, 2) + 2
        lo = np.minimum(2, bins_a[:, d])
        hi = np.minimum(2, nslices[d] - 1 - bins_a[:, d])
        out[:, d] = np.where(valid, (o | (lo << 3) | (hi << 5)).astype(np.uint8), 0xFF)
    out[:, 6] = exact.astype(np.uint8)
    out[:, 7] = 0
    return out


def _ranges(lab: np.ndarray):
    k0 = 2 - ((lab >> 3) & 3).astype(np.int64)
    k1 = 2 + ((lab >> 5) & 3).astype(np.int64)
    return k0, k1


def loss_and_grad(params: np.ndarray, X: np.ndarray, L: np.ndarray, emulate: bool = True):
    """(mean loss, gradient vector) in float64; with emulate, BF16 rounding where the GPU rounds."""
    p = unpack(params)
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    X = np.asarray(X, np.float64)
    B = X.shape[0]
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    if emulate:
        # the GPU's FP32 epilogues: accumulators are FP32, bias added in FP32, then rounded
        f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    else:
        f32 = lambda a: a
    Z1 = f32(f32(X @ W1.T) + p["b1"])
    H1 = r(np.maximum(Z1, 0))
    Z2 = f32(f32(H1 @ W2.T) + p["b2"])
    H2 = r(np.maximum(Z2, 0))
    Z3 = f32(f32(H2 @ W3.T) + p["b3"])
    G = np.zeros_like(Z3)
    loss = 0.0
    for d in range(DIMS):
        lab = L[:, d]
        used = lab != 0xFF
        if not used.any():
            continue
        k0, k1 = _ranges(lab)
        z = Z3[:, d * CLASSES:(d + 1) * CLASSES]
        ks = np.arange(CLASSES)[None, :]
        valid = (ks >= k0[:, None]) & (ks <= k1[:, None]) & used[:, None]
        zm = np.where(valid, z, -np.inf)
        m = np.max(np.where(used[:, None], zm, 0), axis=1)
        e = np.where(valid, np.exp(np.where(valid, z - m[:, None], 0)), 0)
        s = e.sum(axis=1)
        s = np.where(used, s, 1)
        y = np.where(used, lab & 7, 0).astype(np.int64)
        sm = e / s[:, None]
        onehot = (ks == y[:, None]) & used[:, None]
        G[:, d * CLASSES:(d + 1) * CLASSES] = np.where(used[:, None], (sm - onehot) / B, 0)
        zy = z[np.arange(B), y]
        loss += float(np.sum(np.where(used, -(zy - m - np.log(s)), 0)))
    dZ3 = r(G)
    gW3 = dZ3.T @ H2
    gb3 = dZ3.sum(axis=0)
    dZ2 = r(np.where(H2 > 0, dZ3 @ W3, 0))
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(axis=0)
    dZ1 = r(np.where(H1 > 0, dZ2 @ W2, 0))
    gW1 = dZ1.T @ X
    gb1 = dZ1.sum(axis=0)
    grad = pack(dict(W1=gW1, b1=gb1, W2=gW2, b2=gb2, W3=gW3, b3=gb3))
    return loss / B, grad


def forward(params: np.ndarray, X: np.ndarray, emulate: bool = True) -> np.ndarray:
    p = unpack(params)
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    f32 = (lambda a: np.asarray(a, np.float32).astype(np.float64)) if emulate else (lambda a: a)
    X = np.asarray(X, np.float64)
    H1 = r(np.maximum(f32(f32(X @ r(p["W1"]).T) + p["b1"]), 0))
    H2 = r(np.maximum(f32(f32(H1 @ r(p["W2"]).T) + p["b2"]), 0))
    return f32(f32(H2 @ r(p["W3"]).T) + p["b3"])


def topk_cells(logits: np.ndarray, bins: np.ndarray, nslices, k: int = TOPK):
    """Exact top-k offset combinations (by enumeration) of one patch's factorised distribution:
    list of (log-probability, offsets tuple in -2..+2)."""
    G = len(nslices)
    lps = []
    for d in range(G):
        z = np.asarray(logits[d * CLASSES:(d + 1) * CLASSES], np.float64)
        ok = np.array([0 <= bins[d] + o - 2 < nslices[d] for o in range(CLASSES)])
        m = z[ok].max()
        ls = m + np.log(np.exp(z[ok] - m).sum())
        lps.append([(z[o] - ls) if ok[o] else -np.inf for o in range(CLASSES)])
    combos = []
    for offs in itertools.product(range(CLASSES), repeat=G):
        s = sum(lps[d][o] for d, o in enumerate(offs))
        if np.isfinite(s):
            combos.append((s, tuple(o - 2 for o in offs)))
    combos.sort(key=lambda t: -t[0])
    return combos[:k]
