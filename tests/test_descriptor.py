"""Descriptor mode (is_descriptor): tables and queries over caller-supplied descriptor images.

The reference builds the table from the descriptors themselves (get_padded_descriptor,
patchtable.h:2498-2507) and scores every candidate with patch_dist_approx (patchtable.h:376-437)
instead of the RGB patch SSD.  Bars: table, partition and k-coherence set bit-exact with the
oracle (itself pinned to the reference by the golden digests); every NNF_DIST bit-exact with
patch_dist_approx of the returned match; mean distance at most 1% above the reference's."""
import numpy as np
import pytest

import patchtable_b200 as ptb
from oracle.oracle import mean_dist
from patchtable_b200 import synth

from tests.conftest import srand_all
from tests.test_gpu_parity import GOLDEN, MEAN_DIST_SLACK

pytestmark = pytest.mark.gpu


def padded(x, params):
    """The padded descriptor image the reference builds (zeros around an unpadded input)."""
    if params.descriptor_padded:
        return np.ascontiguousarray(x, np.float32)
    h, w, c = x.shape
    out = np.zeros((h + 14, w + 14, c), np.float32)
    out[7:7 + h, 7:7 + w] = x
    return out


def approx_dist(av, bv, nd):
    """patch_dist_approx over rows of vectors, in float32 with its lane order (the vectors carry
    at least four floats; with 3 dimensions the fourth takes part, as in the reference)."""
    d = (av[:, :max(nd, 4)] - bv[:, :max(nd, 4)]).astype(np.float32)
    d = (d * d).astype(np.float32)
    lanes = d[:, :4].copy()
    if nd in (8, 12, 16):
        for n in range(1, nd // 4):
            lanes = (lanes + d[:, 4 * n:4 * n + 4]).astype(np.float32)
        return ((lanes[:, 0] + lanes[:, 1]) + lanes[:, 2]) + lanes[:, 3]
    s = ((lanes[:, 0] + lanes[:, 1]) + lanes[:, 2]) + lanes[:, 3]
    for i in range(4, nd):
        s = (s + d[:, i]).astype(np.float32)
    return s


def check_desc_nnf(params, a, b, ann):
    """Matches inside b's patch grid, integral, and NNF_DIST == patch_dist_approx exactly."""
    A, B = padded(a, params), padded(b, params)
    nd = a.shape[2]
    eh, ew = ann.shape[:2]
    beh, bew = B.shape[0] - 14, B.shape[1] - 14
    bx, by = ann[..., 0], ann[..., 1]
    assert (bx == np.round(bx)).all() and (by == np.round(by)).all()
    assert (bx >= 0).all() and (bx < bew).all() and (by >= 0).all() and (by < beh).all()
    Af = A.reshape(-1)
    Bf = B.reshape(-1)
    ys, xs = np.mgrid[0:eh, 0:ew]
    ia = ((ys + 7) * A.shape[1] + xs + 7).ravel() * nd
    ib = ((by.astype(int) + 7) * B.shape[1] + bx.astype(int) + 7).ravel() * nd
    k = np.arange(max(nd, 4))
    av = Af[ia[:, None] + k[None, :]]
    bv = Bf[ib[:, None] + k[None, :]]
    want = approx_dist(av, bv, nd)
    assert np.array_equal(ann[..., 2].ravel().astype(np.float32), want)


@pytest.mark.parametrize("case", GOLDEN["desc"], ids=[c["name"] for c in GOLDEN["desc"]])
def test_descriptor_mode_build_and_query(gpu, oracle, libc, case):
    a, b = synth.descriptor_pair(case["h"], case["w"], case["c"], case["seed"])
    p = ptb.PatchTableParams(case["switches"])
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    assert gt.shape()[0] == case["nslices"] == ot.shape()[0]
    assert gt.add_count() == ot.add_count()
    for d in range(len(case["nslices"])):
        po, pg = ot.partition(d), gt.partition(d)
        for k in po:
            assert np.array_equal(po[k], pg[k]), (d, k)
    assert np.array_equal(gt.table(), ot.table())
    if p.kcoherence > 0:
        kg, ko = gt.kcoherence(), ot.kcoherence()
        assert np.array_equal(kg[0], ko[0]) and np.array_equal(kg[1], ko[1])
    ann = gt.lookup(a)
    check_desc_nnf(p, a, b, ann)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * case["mean_dist"], (mean_dist(ann), case["mean_dist"])


def test_descriptor_mode_three_channels(gpu, oracle, libc):
    """3 channels: the fourth lane reads the next pixel's first channel (zero beyond the last
    column) on both sides."""
    a, b = synth.descriptor_pair(40, 45, 3, 47)
    p = ptb.PatchTableParams("-limit 0.05 -kcoherence 2 -is_descriptor 1")
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    assert np.array_equal(gt.table(), ot.table())
    kg, ko = gt.kcoherence(), ot.kcoherence()
    assert np.array_equal(kg[0], ko[0]) and np.array_equal(kg[1], ko[1])
    ann = gt.lookup(a)
    check_desc_nnf(p, a, b, ann)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * mean_dist(ot.lookup(a))


def test_reference_test_descriptor_known_answer(gpu, libc):
    """The reference's own test_descriptor (patchtable_main.cpp:174-233): 400x300x8 uniform
    random descriptors; the full table, a 6-dimensional grid, then 6-channel inputs, each scored
    with the double-precision distance over all 8 channels (recompute_mean_dist<1>,
    patchtable_main.cpp:103-172).  It passes when the three means increase and the first is
    below 0.77."""
    rng = np.random.default_rng(9)
    a0 = rng.random((300, 400, 8), dtype=np.float32)
    b0 = rng.random((300, 400, 8), dtype=np.float32)
    dl = []
    for reduce in range(3):
        p = ptb.PatchTableParams("")
        p.is_descriptor = 1
        a, b = a0, b0
        if reduce >= 1:
            p.grid_ndims = 6
        if reduce == 2:
            p.ndims = 6
            a, b = np.ascontiguousarray(a0[..., :6]), np.ascontiguousarray(b0[..., :6])
        srand_all(libc, 1)
        t = ptb.PatchTable(p, b)
        ann = t.lookup(a)
        assert ann.shape == (300, 400, 3)
        bx, by = ann[..., 0].astype(int), ann[..., 1].astype(int)
        assert (bx >= 0).all() and (bx < 400).all() and (by >= 0).all() and (by < 300).all()
        diff = a0.astype(np.float64) - b0.astype(np.float64)[by, bx]
        dl.append(float(np.sqrt((diff * diff).sum(axis=2)).mean()))
        t.close()
    assert dl[0] < dl[1] < dl[2] and dl[0] < 0.77, dl


def test_descriptor_mode_device_and_temporal(gpu, libc):
    """The device entry points take the descriptor image as is; a lookup seeded with its own
    previous field never gets worse."""
    import torch
    a, b = synth.descriptor_pair(70, 90, 8, 48)
    p = ptb.PatchTableParams("-limit 0.3 -kcoherence 2 -is_descriptor 1")
    srand_all(libc, 1)
    t = ptb.PatchTable(p, b)
    host = t.lookup(a)
    da = torch.from_numpy(a).cuda()
    dann = torch.empty(host.shape, dtype=torch.float64, device="cuda")
    t.lookup_device(da.data_ptr(), a.shape[0], a.shape[1], dann.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(dann.cpu().numpy(), host)
    again = t.lookup(a, ann_prev=host)
    check_desc_nnf(p, a, b, again)
    assert (again[..., 2] <= host[..., 2]).all()


def test_descriptor_mode_unsupported_paths(gpu, tmp_path):
    a, b = synth.descriptor_pair(30, 40, 8, 49)
    p = ptb.PatchTableParams("-limit 0.1 -is_descriptor 1")
    t = ptb.PatchTable(p, b)
    for call in (lambda: t.lookup_batch([a]), lambda: t.save(str(tmp_path / "t.bin"))):
        with pytest.raises(ptb.PatchTableError) as e:
            call()
        assert e.value.status == 5
    with pytest.raises(ptb.PatchTableError):
        ptb.PatchTable(ptb.PatchTableParams("-limit 0.1 -is_descriptor 1"), np.zeros((20, 20, 2), np.float32))
