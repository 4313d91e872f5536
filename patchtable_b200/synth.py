"""Seeded synthetic image pairs and PFM I/O.

The reference benchmarks on photo pairs (``vidpairs``, ``one_vs_many``) that are not shipped
with it (patchtable/bench.py:15,79,83).  These generators stand in for them with the shapes,
sizes and value ranges of those workloads: float32 RGB in [0, 1], row-major H x W x 3.

* ``image_a``: 4 octaves of value noise (base period 64 px; period and amplitude halve per
  octave; smoothstep-bilinear lattice, independent per channel, normalised by 1.875), then 20
  axis-aligned rectangles of uniform random colour (origin uniform in the image, sides uniform in
  [8, min(W, H)/4]), clamped to [0, 1].
* ``warp``: a smooth random flow (2 channels of N(0, 1) noise, Gaussian-filtered with sigma 16 px,
  scaled so that its largest vector is 16 px long), bilinear sampling with edge clamp, plus
  N(0, 0.02) noise per channel, clamped to [0, 1].

All randomness comes from ``numpy.random.Generator(PCG64(seed))``.
"""
from __future__ import annotations

import numpy as np

__all__ = ["image_a", "warp", "pair", "crop", "read_pfm", "write_pfm", "batch_sizes"]


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(int(seed)))


def _value_noise(h: int, w: int, rng: np.random.Generator) -> np.ndarray:
    out = np.zeros((h, w, 3), np.float64)
    yy = np.arange(h, dtype=np.float64)[:, None]
    xx = np.arange(w, dtype=np.float64)[None, :]
    period, amp = 64.0, 1.0
    for _ in range(4):
        gh = int(np.floor((h - 1) / period)) + 2
        gw = int(np.floor((w - 1) / period)) + 2
        lattice = rng.random((gh, gw, 3))
        u, v = xx / period, yy / period
        i, j = np.floor(u).astype(np.int64), np.floor(v).astype(np.int64)
        fx, fy = u - i, v - j
        sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
        i = np.broadcast_to(i, (h, w))
        j = np.broadcast_to(j, (h, w))
        sx = np.broadcast_to(sx, (h, w))[..., None]
        sy = np.broadcast_to(sy, (h, w))[..., None]
        c00, c01 = lattice[j, i], lattice[j, i + 1]
        c10, c11 = lattice[j + 1, i], lattice[j + 1, i + 1]
        top = c00 + (c01 - c00) * sx
        bot = c10 + (c11 - c10) * sx
        out += amp * (top + (bot - top) * sy)
        period *= 0.5
        amp *= 0.5
    return out / 1.875


def image_a(h: int, w: int, seed: int) -> np.ndarray:
    """Value noise plus 20 random rectangles, float32 H x W x 3 in [0, 1]."""
    rng = _rng(seed)
    img = _value_noise(h, w, rng)
    smax = max(8, min(w, h) // 4)
    for _ in range(20):
        x0, y0 = int(rng.integers(0, w)), int(rng.integers(0, h))
        rw, rh = int(rng.integers(8, smax + 1)), int(rng.integers(8, smax + 1))
        img[y0:y0 + rh, x0:x0 + rw, :] = rng.random(3)
    return np.clip(img, 0.0, 1.0).astype(np.float32)


def _gaussian_1d(sigma: float) -> np.ndarray:
    r = int(np.ceil(3 * sigma))
    t = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (t / sigma) ** 2)
    return k / k.sum()


def _blur(img: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian blur with reflected borders (2-D float64 input)."""
    k = _gaussian_1d(sigma)
    r = (len(k) - 1) // 2
    out = img
    for axis in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[axis] = (r, r)
        p = np.pad(out, pad, mode="symmetric")
        acc = np.zeros_like(out)
        n = out.shape[axis]
        for t, kv in enumerate(k):
            sl = [slice(None), slice(None)]
            sl[axis] = slice(t, t + n)
            acc += kv * p[tuple(sl)]
        out = acc
    return out


def warp(img: np.ndarray, seed: int, max_disp: float = 16.0, sigma: float = 16.0,
         noise: float = 0.02) -> np.ndarray:
    """Warp by a smooth random flow, add Gaussian noise, clamp. Returns float32 H x W x 3."""
    rng = _rng(seed)
    h, w, _ = img.shape
    fx = _blur(rng.standard_normal((h, w)), sigma)
    fy = _blur(rng.standard_normal((h, w)), sigma)
    mag = np.sqrt(fx * fx + fy * fy).max()
    s = max_disp / mag if mag > 0 else 0.0
    fx *= s
    fy *= s
    xs = np.clip(np.arange(w)[None, :] + fx, 0, w - 1)
    ys = np.clip(np.arange(h)[:, None] + fy, 0, h - 1)
    x0 = np.minimum(np.floor(xs).astype(np.int64), w - 2 if w > 1 else 0)
    y0 = np.minimum(np.floor(ys).astype(np.int64), h - 2 if h > 1 else 0)
    tx = (xs - x0)[..., None]
    ty = (ys - y0)[..., None]
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    src = img.astype(np.float64)
    top = src[y0, x0] * (1 - tx) + src[y0, x1] * tx
    bot = src[y1, x0] * (1 - tx) + src[y1, x1] * tx
    out = top * (1 - ty) + bot * ty
    out += rng.normal(0.0, noise, out.shape)
    return np.clip(out, 0.0, 1.0).astype(np.float32)


def pair(h: int, w: int, seed: int):
    """(a, b): b is a warp of a (flow seed = seed + 1000003)."""
    a = image_a(h, w, seed)
    b = warp(a, seed + 1000003)
    return a, b


def descriptor_pair(h: int, w: int, channels: int = 8, seed: int = 0):
    """A pair of h x w x channels descriptor images for descriptor mode (is_descriptor): fixed
    random linear features of the 3x3 grid of pixels 2 apart around each pixel (edge-replicated)
    of ``pair(h, w, seed)``, so b's descriptors follow a's under the same warp."""
    a, b = pair(h, w, seed)
    rng = _rng(seed + 12345)
    taps = [(dy, dx) for dy in (-2, 0, 2) for dx in (-2, 0, 2)]
    proj = (rng.standard_normal((channels, 3 * len(taps))) / np.sqrt(3 * len(taps))).astype(np.float32)

    def feat(img):
        pad = np.pad(img, ((2, 2), (2, 2), (0, 0)), mode="edge")
        stack = np.concatenate([pad[2 + dy:2 + dy + h, 2 + dx:2 + dx + w] for dy, dx in taps], axis=2)
        return np.ascontiguousarray(stack @ proj.T, dtype=np.float32)
    return feat(a), feat(b)


def crop(img: np.ndarray, h: int, w: int, seed: int) -> np.ndarray:
    """Random h x w crop (clamped to the image)."""
    rng = _rng(seed)
    H, W, _ = img.shape
    h, w = min(h, H), min(w, W)
    y0 = int(rng.integers(0, H - h + 1))
    x0 = int(rng.integers(0, W - w + 1))
    return np.ascontiguousarray(img[y0:y0 + h, x0:x0 + w])


def batch_sizes(n: int, lo: int, hi: int, seed: int):
    """n (h, w) pairs with each side uniform in [lo, hi]."""
    rng = _rng(seed)
    return [(int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1))) for _ in range(n)]


def uneven_batch(n: int = 64, lo: int = 128, hi: int = 2048, seed: int = 4000):
    """Uneven query batch against one table: (table image, [query images]).

    A 2048 x 2048 base image (seed); the table image is a 1080 x 1920 crop of it; query i is an
    (h_i, w_i) crop, sides uniform in [lo, hi] (seed + i), of the base warped once by the smooth
    random flow (seed + 1).  Warping the base once, instead of every crop, keeps generation to a
    few seconds; every query is still a warped view of the scene the table indexes."""
    base = image_a(2048, 2048, seed)
    wb = warp(base, seed + 1)
    table = crop(base, 1080, 1920, seed)
    queries = [crop(wb, h, w, seed + i) for i, (h, w) in enumerate(batch_sizes(n, lo, hi, seed))]
    return table, queries


def one_vs_many(n: int = 10, lo: int = 256, hi: int = 2048, seed: int = 3000, qh: int = 768, qw: int = 1024):
    """One query against a database of n images packed into one atlas.

    Returns (query, atlas, allowed, boxes): the query is a qh x qw crop of a 2048 x 2048 base image
    (seed); database image i is a crop, sides uniform in [lo, hi] (seed + 1 + i), of the base warped
    once (seed + 1).  The images are packed on shelves (tallest first) into one atlas; allowed
    marks with 1 the patches that lie inside one image (seam-straddling and padding patches get 0),
    and boxes lists each image's (y, x, h, w) in the atlas."""
    base = image_a(2048, 2048, seed)
    wb = warp(base, seed + 1)
    query = crop(base, qh, qw, seed)
    sizes = batch_sizes(n, lo, hi, seed + 1)
    db = [crop(wb, h, w, seed + 1 + i) for i, (h, w) in enumerate(sizes)]
    order = sorted(range(n), key=lambda i: -db[i].shape[0])
    width = max(4096, max(x.shape[1] for x in db))
    boxes = [None] * n
    y = x = shelf = 0
    for i in order:
        h, w = db[i].shape[:2]
        if x + w > width:
            y, x, shelf = y + shelf, 0, 0
        boxes[i] = (y, x, h, w)
        x += w
        shelf = max(shelf, h)
    H = y + shelf
    atlas = np.zeros((H, width, 3), np.float32)
    allowed = np.zeros((H - 7, width - 7), np.int32)
    for i, (y0, x0, h, w) in enumerate(boxes):
        atlas[y0:y0 + h, x0:x0 + w] = db[i]
        allowed[y0:y0 + h - 7, x0:x0 + w - 7] = 1
    return query, atlas, allowed, boxes


def write_pfm(path: str, img: np.ndarray) -> None:
    """3-channel little-endian PFM, rows stored bottom-up (solver/pfm.cpp:50-64)."""
    img = np.asarray(img, np.float32)
    h, w, c = img.shape
    assert c == 3
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.000000\n" % (w, h))
        f.write(np.ascontiguousarray(img[::-1]).astype("<f4").tobytes())


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        kind = f.readline().strip()
        w, h = (int(t) for t in f.readline().split())
        scale = float(f.readline())
        c = 3 if kind == b"PF" else 1
        dt = "<f4" if scale < 0 else ">f4"
        data = np.frombuffer(f.read(w * h * c * 4), dtype=dt).astype(np.float32)
    return np.ascontiguousarray(data.reshape(h, w, c)[::-1])
