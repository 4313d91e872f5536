"""The host lookup of one-pass schedules streams the image through bands of rows (uploads and
downloads overlapped with the kernels).  Its NNF must equal the whole-image device lookup's bit
for bit, for every image shape, band remainder and propagation radius."""
import numpy as np
import pytest

import patchtable_b200 as ptb
from patchtable_b200 import synth

pytestmark = pytest.mark.gpu


def _device(t, a):
    import torch
    h, w = a.shape[:2]
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ann = torch.empty((h - 7, w - 7, 3), dtype=torch.float64, device="cuda")
    t.lookup_device(da.data_ptr(), h, w, ann.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return ann.cpu().numpy()


@pytest.mark.parametrize("h,w,sw", [
    (1080, 1920, "-speed 3 -coherence_spatial 4"),
    (71, 100, "-speed 3 -coherence_spatial 4 -limit 2"),
    (333, 200, "-speed 3 -coherence_spatial 4 -limit 2 -gpu_tile 128"),
    (517, 263, "-speed 3 -coherence_spatial 4 -limit 2 -query_step 2 -gpu_jump 8"),
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


def test_banded_graph_replay_with_page_locked_images(gpu, libc):
    """A page-locked query image seen again with the same sizes and parameters is answered by
    replaying the recorded band graph; a second page-locked image re-points its upload nodes, a
    pageable one is enqueued directly, a parameter change records anew.  Every answer equals the
    device lookup's, and the host threads' count does not change it."""
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
    for img, ref in ((pa, want), (pa, want), (pa, want), (pa2, want2), (pa, want), (a2, want2), (pa, want)):
        out[:] = -1
        t.lookup(img, out=out)
        assert np.array_equal(out, ref)
    p.gpu_tile = 64
    for _ in range(3):
        assert np.array_equal(t.lookup(pa), want)
    old = ptb.set_host_threads(1)
    try:
        assert np.array_equal(t.lookup(pa), want)
    finally:
        ptb.set_host_threads(old)
    assert t.last_transfer() == (a.nbytes, 8 * want.shape[0] * want.shape[1])
    t.close()
