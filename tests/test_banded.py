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
