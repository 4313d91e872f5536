"""Image analogies (patchtable/analogy.cpp) over GPU patch tables, one frame.

The reference's analogy needs OpenCV (its pyramid resize, optical flow), which is absent here, so
its output cannot be reproduced; the pipeline is checked by what an analogy must do: learn a
filter from (a, ap) and apply it to b."""
import numpy as np
import pytest

from patchtable_b200 import analogy, synth

pytestmark = pytest.mark.gpu


def _invert_luma(img):
    yuv = analogy.rgb2yuv(img)
    yuv[..., 0] = 1.0 - yuv[..., 0]
    return analogy.yuv2rgb(yuv)


def test_analogy_learns_a_luminance_inversion(gpu, libc):
    a, b = synth.pair(96, 128, 61)
    ap = _invert_luma(a)
    libc.srand(1)
    bp = analogy.analogy(a, ap, b, "-levels 4 -min_size 24 -limit 0.5")
    assert bp.shape == b.shape and np.isfinite(bp).all()
    want = analogy.rgb2yuv(_invert_luma(b))[..., 0]
    got = analogy.rgb2yuv(bp)[..., 0]
    inner = (slice(8, -8), slice(8, -8))
    err = np.abs(got - want)[inner].mean()
    base = np.abs(analogy.rgb2yuv(b)[..., 0] - want)[inner].mean()
    assert err < 0.1 * base, (err, base)
    # b's chrominance comes back through yuv2rgb, whose constants only nearly invert rgb2yuv
    assert np.allclose(analogy.rgb2yuv(bp)[..., 1:], analogy.rgb2yuv(b)[..., 1:], atol=1e-4)


def test_analogy_switches_and_helpers(gpu, libc):
    ap_params, rest = analogy.parse_switches("-levels 3 -lum_only 0 -ap_weight 0.5 -limit 0.2 -kcoherence 4")
    assert ap_params["levels"] == 3 and ap_params["lum_only"] is False and ap_params["ap_weight"] == 0.5
    assert rest == "-limit 0.2 -kcoherence 4"
    img = synth.pair(60, 80, 3)[0]
    assert np.allclose(analogy.yuv2rgb(analogy.rgb2yuv(img)), img, atol=2e-4)
    sizes = [x.shape[:2] for x in analogy.pyramid(img, 4, 15)]
    assert sizes[0] == (15, 20) and sizes[-1] == (60, 80)
    a, b = synth.pair(72, 90, 62)
    libc.srand(1)
    bp = analogy.analogy(a, a, b, "-levels 3 -min_size 30 -limit 0.2 -lum_only 0")
    # the identity filter rebuilds b from a's patches: far closer to b than a itself (b is a
    # warp of a plus noise, so a exact copy is not expected)
    assert np.abs(bp - b)[8:-8, 8:-8].mean() < 0.5 * np.abs(a - b)[8:-8, 8:-8].mean()
