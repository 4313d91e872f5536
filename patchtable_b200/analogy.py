"""Image analogies on GPU patch tables: the reference's `patchtable analogy a ap b out`
(patchtable/analogy.cpp:804-1162), for one frame.

Given a pair (a, ap) and a target b, synthesise bp so that bp relates to b as ap relates to a
(Hertzmann et al.'s image analogies, the reference's main in-repo caller of PatchTable):

* all three images go to YUV and a, ap get b's luminance mean and spread (lum_remap,
  analogy.cpp:279-297);
* pyramids of `levels` sizes from `min_size` rows up to the full image, spaced geometrically
  (Pyramid, analogy.cpp:229-258);
* per level, a descriptor-mode table over the composite descriptor [GCK(a_Y), ap_weight x
  GCK(ap_Y)] with ndims/2 Walsh-Hadamard channels each, padded like gck's output
  (get_composite_descriptor, analogy.cpp:299-326; descriptor_padded), and at the coarsest level
  an image-mode table of a itself with ndims/2 channels (analogy.cpp:866-893);
* synthesis from coarse to fine: `correction_iters` rounds of lookup (the first one at the
  coarsest level through a's own table, later ones with the composite of (b, current bp) and the
  previous field as ann_prev) and vote, the overlapping patches of ap averaged into bp's
  luminance (vote, analogy.cpp:362-491), then bp upsampled to the next level;
* bp takes b's chrominance back (lum_only) and returns to RGB.

The lookups are the library's GPU tables; the remaining host steps are small numpy passes.  The
reference resizes with OpenCV's Lanczos filter after a Gaussian prefilter (solver/array.h:3221);
OpenCV is not available here, so levels are resampled with separable area averaging when
shrinking and bilinear interpolation when growing.  Video input (optical flow, shot detection,
temporal NNF correction) is not covered.
"""
from __future__ import annotations

import numpy as np

import patchtable_b200 as ptb

DEFAULTS = dict(min_size=15, levels=8, correction_iters=2, vote_overlapping=True, lum_only=True,
                upweight_coherence=0.0, ap_weight=1.0, fine_levels=2, fine_coherence_spatial=-1.0,
                fine_upweight_coherence=-1.0)          # AnalogyParams::set_defaults, analogy.cpp:122-171
_INT_KEYS = ("min_size", "levels", "correction_iters", "fine_levels")
_BOOL_KEYS = ("vote_overlapping", "lum_only")


def parse_switches(switches: str):
    """Analogy switches (analogy.cpp:66-118) and the remaining PatchTable switches."""
    ap = dict(DEFAULTS)
    rest = []
    toks = switches.split()
    i = 0
    while i < len(toks):
        key = toks[i].lstrip("-")
        if toks[i].startswith("-") and key in ap and i + 1 < len(toks):
            v = toks[i + 1]
            ap[key] = int(v) if key in _INT_KEYS else (bool(int(v)) if key in _BOOL_KEYS else float(v))
            i += 2
            continue
        rest.append(toks[i])
        i += 1
    return ap, " ".join(rest)


def rgb2yuv(img):
    """ARRAY_RGB2YUV (solver/array.h:1116-1127): double constants, float pixels."""
    x = img.astype(np.float64)
    r, g, b = x[..., 0], x[..., 1], x[..., 2]
    return np.stack([0.299 * r + 0.587 * g + 0.114 * b, -0.14713 * r + -0.28886 * g + 0.436 * b,
                     0.615 * r + -0.51499 * g + -0.10001 * b], axis=-1).astype(np.float32)


def yuv2rgb(img):
    """Array::yuv2rgb (solver/array.h:1143-1155)."""
    x = img.astype(np.float64)
    y, u, v = x[..., 0], x[..., 1], x[..., 2]
    return np.stack([y + 1.13983 * v, y + -0.39465 * u + -0.58060 * v, y + 2.03211 * u], axis=-1).astype(np.float32)


def lum_remap(a, ap, b):
    """a and ap luminance mapped to b's mean and standard deviation, clamped to [0, 1]."""
    def ms(x):
        c = x[..., 0].astype(np.float64)
        m = c.mean()
        return m, np.sqrt((c * c).mean() - m * m)
    am, asg = ms(a)
    bm, bsg = ms(b)
    for x in (a, ap):
        x[..., 0] = np.clip(bsg / asg * (x[..., 0] - am) + bm, 0.0, 1.0)


def _resize_axis(x, n, axis):
    m = x.shape[axis]
    if n == m:
        return x
    x = np.moveaxis(x, axis, 0).astype(np.float64)
    if n < m:                                   # area average over each output cell
        edges = np.linspace(0.0, m, n + 1)
        cs = np.concatenate([np.zeros((1,) + x.shape[1:]), np.cumsum(x, axis=0)])

        def at(e):
            i = np.minimum(np.floor(e).astype(int), m - 1)
            f = (e - i).reshape((-1,) + (1,) * (x.ndim - 1))
            return cs[i] + f * x[i]
        out = (at(edges[1:]) - at(edges[:-1])) / (edges[1:] - edges[:-1]).reshape((-1,) + (1,) * (x.ndim - 1))
    else:                                       # bilinear, pixel centres aligned
        pos = np.clip((np.arange(n) + 0.5) * m / n - 0.5, 0, m - 1)
        i0 = np.floor(pos).astype(int)
        i1 = np.minimum(i0 + 1, m - 1)
        f = (pos - i0).reshape((-1,) + (1,) * (x.ndim - 1))
        out = x[i0] * (1 - f) + x[i1] * f
    return np.moveaxis(out, 0, axis)


def resize(img, w, h):
    """Image resampled to w x h (stand-in for the reference's imresize)."""
    return np.ascontiguousarray(_resize_axis(_resize_axis(img, h, 0), w, 1), dtype=np.float32)


def pyramid(img, levels, min_size):
    """Level i has height exp(log(min_size) + (log(H) - log(min_size)) * i / (levels - 1))."""
    H, W = img.shape[:2]
    out = []
    for i in range(levels):
        t = i / (levels - 1.0) if levels > 1 else 1.0
        h = np.exp(np.log(min_size) + (np.log(H) - np.log(min_size)) * t)
        w = W / H * h
        out.append(resize(img, int(w + 0.5), int(h + 0.5)))
    return out


def _gck_luma(img, n):
    """Padded (h+7) x (w+7) x n GCK descriptor of the luminance (gck with nchroma 0); the
    border, which no patch of a padded descriptor reads, is zero."""
    p = ptb.PatchTableParams("-ndims %d -nchroma 0 -colorspace rgb" % n)
    h, w = img.shape[:2]
    out = np.zeros((h + 7, w + 7, n), np.float32)
    out[7:h, 7:w] = ptb.descriptor(p, img)
    return out


def composite(a, ap, ndims, ap_weight):
    """get_composite_descriptor: [GCK(a_Y), ap_weight x GCK(ap_Y)]."""
    da = _gck_luma(a, ndims // 2)
    dp = _gck_luma(ap, ndims // 2)
    return np.ascontiguousarray(np.concatenate([da, np.float32(ap_weight) * dp], axis=-1))


def vote(bnn, a, upweight_coherence=0.0, overlapping=True, lum_only=True):
    """bp from the patches of a that bnn points to: each pixel the (weighted) mean of the
    patches covering it (vote, analogy.cpp:362-491)."""
    eh, ew = bnn.shape[:2]
    h, w = eh + 7, ew + 7
    ax = np.clip(bnn[..., 0].astype(int), 0, a.shape[1] - 8)
    ay = np.clip(bnn[..., 1].astype(int), 0, a.shape[0] - 8)
    nc = 1 if lum_only else 3
    out = np.zeros((h, w, 3), np.float32)
    if not overlapping:
        for dy in range(8):
            for dx in range(8):
                out[dy:dy + eh, dx:dx + ew, :nc] = a[ay + dy, ax + dx, :nc]
        return out
    wpatch = np.ones((eh, ew))
    if upweight_coherence:
        n = np.zeros((eh, ew), int)           # coherent neighbours (coherence_weight, analogy.cpp:328-360)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dx == 0 and dy == 0:
                    continue
                ys, xs = np.mgrid[0:eh, 0:ew]
                yp, xp = ys + dy, xs + dx
                ok = (yp >= 0) & (yp < eh) & (xp >= 0) & (xp < ew)
                ypc, xpc = np.clip(yp, 0, eh - 1), np.clip(xp, 0, ew - 1)
                n += ok & (bnn[ypc, xpc, 0].astype(int) == ax + dx) & (bnn[ypc, xpc, 1].astype(int) == ay + dy)
        wpatch = 1e-6 + np.power(n.astype(np.float64), upweight_coherence)
    acc = np.zeros((h, w, nc))
    wsum = np.zeros((h, w))
    for dy in range(8):
        for dx in range(8):
            acc[dy:dy + eh, dx:dx + ew] += a[ay + dy, ax + dx, :nc] * wpatch[..., None]
            wsum[dy:dy + eh, dx:dx + ew] += wpatch
    out[..., :nc] = acc / wsum[..., None]
    return out


def analogy(a_rgb, ap_rgb, b_rgb, switches: str = ""):
    """bp (RGB, b's size) such that bp : b :: ap : a."""
    ap_params, table_sw = parse_switches(switches)
    a, ap, b = rgb2yuv(a_rgb), rgb2yuv(ap_rgb), rgb2yuv(b_rgb)
    lum_remap(a, ap, b)
    base = "-ndims 8 -coherence_spatial 80 -coherence_temporal 1 -colorspace rgb " + table_sw   # analogy.cpp:847-853
    p = ptb.PatchTableParams(base)
    if p.ndims % 2:
        raise ptb.PatchTableError(1, "analogy: ndims must be even")
    p.nchroma = 0
    p.descriptor_padded = 1
    nd = p.ndims
    p0 = ptb.PatchTableParams(base)                    # p0: half the dimensions, on a itself (analogy.cpp:862-863)
    p0.ndims, p0.nchroma, p0.descriptor_padded = nd // 2, 0, 0
    L, ms = ap_params["levels"], ap_params["min_size"]
    a_pyr, ap_pyr, b_pyr = pyramid(a, L, ms), pyramid(ap, L, ms), pyramid(b, L, ms)
    p.is_descriptor = 1
    tables = [ptb.PatchTable(p, composite(a_pyr[i], ap_pyr[i], nd, ap_params["ap_weight"])) for i in range(L)]
    a0 = ptb.PatchTable(p0, a_pyr[0])
    cs0 = p.coherence_spatial
    bp = None
    for level in range(L):
        p.coherence_spatial = cs0
        upw = ap_params["upweight_coherence"]
        if level >= L - ap_params["fine_levels"]:
            if ap_params["fine_coherence_spatial"] >= 0:
                p.coherence_spatial = ap_params["fine_coherence_spatial"]
            if ap_params["fine_upweight_coherence"] >= 0:
                upw = ap_params["fine_upweight_coherence"]
        bnn = None
        for it in range(ap_params["correction_iters"]):
            prev = bnn
            if level == 0 and it == 0:
                bnn = a0.lookup(b_pyr[0])
            else:
                bnn = tables[level].lookup(composite(b_pyr[level], bp, nd, ap_params["ap_weight"]), ann_prev=prev)
            bp = vote(bnn, ap_pyr[level], upw, ap_params["vote_overlapping"], ap_params["lum_only"])
        if level + 1 < L:
            nxt = b_pyr[level + 1]
            bp = resize(bp, nxt.shape[1], nxt.shape[0])
    for t in tables + [a0]:
        t.close()
    if ap_params["lum_only"]:
        bp[..., 1:] = b[..., 1:]
    return yuv2rgb(bp)


def main(argv=None):
    """python -m patchtable_b200.analogy a.pfm ap.pfm b.pfm out.pfm [switches]"""
    import sys
    from patchtable_b200 import synth
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 4:
        print(main.__doc__)
        return 1
    a, ap, b = (synth.read_pfm(f) for f in argv[:3])
    synth.write_pfm(argv[3], analogy(a, ap, b, " ".join(argv[4:])))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
