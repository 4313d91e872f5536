"""The host lookup of one-pass schedules streams the image through bands of rows (uploads and
downloads overlapped with the kernels).  Its NNF must equal the whole-image device lookup's bit
for bit, for every image shape, band remainder and propagation radius."""
import numpy as np
import pytest

import patchtable_b200 as ptb
from patchtable_b200 import synth

pytestmark = pytest.mark.gpu


def _device(t, a):
    """The whole-image launch sequence, through the diagnostic and the device entry points."""
    import torch
    h, w = a.shape[:2]
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ann = torch.empty((h - 7, w - 7, 3), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    t.lookup_profile(da.data_ptr(), h, w, ann.data_ptr(), st)
    whole = ann.cpu().numpy()
    ann.fill_(-1)
    t.lookup_device(da.data_ptr(), h, w, ann.data_ptr(), st)
    torch.cuda.synchronize()
    assert np.array_equal(ann.cpu().numpy(), whole)
    return whole


@pytest.mark.parametrize("h,w,sw", [
    (1080, 1920, "-speed 3 -coherence_spatial 4"),
    (71, 100, "-speed 3 -coherence_spatial 4 -limit 2"),
    (333, 200, "-speed 3 -coherence_spatial 4 -limit 2 -gpu_tile 128"),
    (517, 263, "-speed 3 -coherence_spatial 4 -limit 2 -query_step 2 -gpu_jump 8"),
    (300, 411, "-speed 3 -coherence_spatial 4 -limit 2 -gpu_kc_max -1"),
])
def test_banded_host_lookup_equals_device(gpu, libc, h, w, sw):
    a, b = synth.pair(h, w, 90 + h)
    p = ptb.PatchTableParams(sw)
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    p.gpu_prop_passes = 1
    if p.gpu_pull_max == 0 and h > 1000:
        p.gpu_pull_max = 1
    host = t.lookup(a)
    dev = _device(t, a)
    assert np.array_equal(host, dev)
    pinned = np.empty_like(host)
    t.lookup(a, out=pinned)
    assert np.array_equal(pinned, dev)
    for bands in (1, 5, 40):                 # the band count changes only the overlap
        p.gpu_bands = bands
        assert np.array_equal(t.lookup(a), dev), bands


def test_banded_with_allowed_mask(gpu, libc):
    a, b = synth.pair(200, 180, 77)
    allowed = np.ones((193, 173), np.int32)
    allowed[:, 80:90] = 0
    p = ptb.PatchTableParams("-speed 3 -coherence_spatial 4 -limit 2")
    libc.srand(1)
    t = ptb.PatchTable(p, b, allowed_patches=allowed)
    p.gpu_prop_passes = 1
    host = t.lookup(a)
    assert np.array_equal(host, _device(t, a))
    assert np.all(allowed[host[..., 1].astype(int), host[..., 0].astype(int)] == 1)


def test_banded_repeated_lookups_page_locked_and_pageable(gpu, libc):
    """Repeated host lookups of page-locked and pageable images, with the packed download widened
    by one or several host threads or the float64 records downloaded as they are: every answer
    equals the device lookup's, and the transfer accounting matches the mode."""
    import torch
    a, b = synth.pair(300, 420, 81)
    a2 = synth.image_a(300, 420, 82)
    p = ptb.PatchTableParams("-speed 3 -coherence_spatial 4 -limit 2")
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    p.gpu_prop_passes, p.gpu_pull_max = 1, 1
    want, want2 = _device(t, a), _device(t, a2)
    pa = torch.from_numpy(a).pin_memory().numpy()
    pa2 = torch.from_numpy(a2).pin_memory().numpy()
    out = torch.empty(want.shape, dtype=torch.float64).pin_memory().numpy()
    old = ptb.set_host_threads(0)
    try:
        for threads in (0, 1, 3, -1):
            ptb.set_host_threads(threads)
            for img, ref in ((pa, want), (pa, want), (pa2, want2), (a2, want2), (pa, want)):
                out[:] = -1
                t.lookup(img, out=out)
                assert np.array_equal(out, ref), threads
            assert np.array_equal(t.lookup(a2), want2)
            per_patch = 24 if threads < 0 else 8
            assert t.last_transfer() == (a.nbytes, per_patch * want.shape[0] * want.shape[1])
    finally:
        ptb.set_host_threads(old)
    t.close()
