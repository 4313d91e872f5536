"""Batched queries (one launch per phase for many images of any sizes) and the allowed-patch mask
of one-vs-many atlas tables.

A batch computes every patch exactly as the single-image query does, so each image's NNF in a
batch must equal its own pt_table_lookup result bit for bit, for every choice of patches per CTA,
through a captured CUDA graph, and through the host entry point pt_table_lookup_batch."""
import numpy as np
import pytest

import patchtable_b200 as ptb
from oracle.oracle import mean_dist
from patchtable_b200 import synth

from tests.test_gpu_parity import MEAN_DIST_SLACK, check_nnf

pytestmark = pytest.mark.gpu

SIZES = [(40, 50), (64, 300), (130, 77), (8, 8), (200, 160), (33, 260), (9, 270)]


def _table(libc, sw="-speed 3 -coherence_spatial 4 -limit 2", h=160, w=200, seed=21):
    a, b = synth.pair(h, w, seed)
    libc.srand(1)
    return ptb.PatchTable(ptb.PatchTableParams(sw), b), b


def _queries(seed0=300):
    return [synth.pair(h, w, seed0 + i)[0] for i, (h, w) in enumerate(SIZES)]


def _device_batch(t, imgs):
    import torch
    qb = t.batch([x.shape[:2] for x in imgs])
    rgb = torch.empty(qb.pixels * 3, dtype=torch.float32, device="cuda")
    for x, o in zip(imgs, qb.pixel_offset):
        rgb[3 * o:3 * o + x.size] = torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()
    ann = torch.full((qb.patches * 3,), -7.0, dtype=torch.float64, device="cuda")
    return qb, rgb, ann


def _split(qb, imgs, ann):
    host = ann.cpu().numpy()
    out = []
    for x, o in zip(imgs, qb.patch_offset):
        eh, ew = x.shape[0] - 7, x.shape[1] - 7
        out.append(host[3 * o:3 * (o + eh * ew)].reshape(eh, ew, 3))
    return out


@pytest.mark.parametrize("sched", [(0, 0, 0), (1, 2, 1), (2, 2, 0), (1, 2, 1, -1), (2, 2, 0, 1)])
def test_batch_equals_per_image(gpu, libc, sched):
    import torch
    t, b = _table(libc)
    t.params.set_schedule(sched)
    imgs = _queries()
    single = [t.lookup(x) for x in imgs]
    host = t.lookup_batch(imgs)
    for s, h in zip(single, host):
        assert np.array_equal(s, h)
    qb, rgb, ann = _device_batch(t, imgs)
    st = torch.cuda.current_stream().cuda_stream
    for tile in (32, 64, 128, 256):
        qb.set_tile(tile)
        ann.fill_(-7.0)
        qb.lookup(rgb.data_ptr(), ann.data_ptr(), st)
        torch.cuda.synchronize()
        for s, got in zip(single, _split(qb, imgs, ann)):
            assert np.array_equal(s, got), tile


def test_batch_graph_replay_and_autotune(gpu, libc):
    import torch
    t, b = _table(libc)
    imgs = _queries(400)
    single = [t.lookup(x) for x in imgs]
    qb, rgb, ann = _device_batch(t, imgs)
    st = torch.cuda.current_stream().cuda_stream
    best, ms = qb.autotune(rgb.data_ptr(), ann.data_ptr(), st)
    assert best in (32, 64, 128, 256) and qb.tile == best
    assert all(v > 0 for v in ms.values())
    qb.capture(rgb.data_ptr(), ann.data_ptr(), st)
    for _ in range(2):                       # two replays in a row: same result each time
        ann.fill_(-7.0)
        qb.replay(st)
        torch.cuda.synchronize()
        for s, got in zip(single, _split(qb, imgs, ann)):
            assert np.array_equal(s, got)


def test_batch_rejects_bad_sizes(gpu, libc):
    t, b = _table(libc)
    with pytest.raises(ptb.PatchTableError):
        t.batch([(7, 100)])
    with pytest.raises(ptb.PatchTableError):
        t.batch([])


def test_atlas_with_allowed_patches(gpu, oracle, libc):
    """One-vs-many: two database images packed side by side into one atlas table; patches that
    straddle the seam are excluded with the allowed mask, and no match may land on them."""
    b1 = synth.pair(150, 120, 31)[1]
    b2 = synth.pair(150, 96, 32)[1]
    atlas = np.ascontiguousarray(np.concatenate([b1, b2], axis=1))
    beh, bew = atlas.shape[0] - 7, atlas.shape[1] - 7
    allowed = np.zeros((beh, bew), np.int32)
    allowed[:, :120 - 7] = 1                 # patches entirely inside b1
    allowed[:, 120:] = 1                     # patches entirely inside b2
    a = synth.pair(150, 120, 31)[0]
    p = ptb.PatchTableParams("-speed 3 -coherence_spatial 4 -limit 2")
    libc.srand(1)
    gt = ptb.PatchTable(p, atlas, allowed_patches=allowed)
    ann = gt.lookup(a)
    check_nnf(oracle, a, atlas, ann)
    xs, ys = ann[..., 0].astype(int), ann[..., 1].astype(int)
    assert np.all(allowed[ys, xs] == 1)
    libc.srand(1)
    ot = oracle.build(p.as_dict(), atlas, allowed=allowed)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * mean_dist(ot.lookup(a))
    qb_ann = gt.lookup_batch([a])[0]
    assert np.array_equal(qb_ann, ann)


@pytest.mark.parametrize("sw", ["-speed 3 -coherence_spatial 4 -limit 2 -colorspace lab",
                                "-speed 3 -limit 2 -colorspace rgb -spatial 1"])
def test_batch_other_colour_spaces_and_search(gpu, libc, sw):
    """The batched descriptor and choose kernels follow the table's colour space and search
    options exactly as the single-image query does."""
    t, b = _table(libc, sw)
    imgs = _queries(500)[:4]
    single = [t.lookup(x) for x in imgs]
    for s, h in zip(single, t.lookup_batch(imgs)):
        assert np.array_equal(s, h)


@pytest.mark.parametrize("sw", ["-speed 3 -do_prop 0 -limit 2", "-speed 3 -prop_iters 0 -limit 2"])
def test_schedules_without_propagation(gpu, oracle, libc, sw):
    """Without propagation the last step is not a pull (the output is written by its own launch)
    and with no iterations the field stays the initial one: batches, device and host lookups all
    agree, and with prop_iters 0 the NNF equals the oracle's initial field exactly."""
    t, b = _table(libc, sw)
    imgs = _queries(700)[:4]
    single = [t.lookup(x) for x in imgs]
    for s, h in zip(single, t.lookup_batch(imgs)):
        assert np.array_equal(s, h)
    if "-prop_iters 0" in sw:
        ot = oracle.build(t.params.as_dict(), b)
        for x, s in zip(imgs, single):
            assert np.array_equal(s, ot.lookup(x))
    else:
        for x, s in zip(imgs, single):
            check_nnf(oracle, x, b, s, sample=300)
