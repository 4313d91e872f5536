"""GPU path vs the CPU oracle (run with -m gpu on a B200).

Bars, per the path's contract:
  * descriptors: within 1e-6 x (sum of the |terms| of the patch's projection) of exact float64
    arithmetic -- a rigorous bound for two 8-term float sums -- and never farther from the oracle
    than the oracle's own float running sums are from exact arithmetic (plus that bound);
  * partition, table after the DT, k-coherence set: bit-exact given the oracle's descriptors;
  * every NNF_DIST: bit-exact with the reference's patch_dist_exact for the returned match, and
    within 1e-5 relative of a float64 recompute;
  * mean NNF distance: at most 1% above the oracle's (propagation order legitimately differs).
"""
import importlib.util
import json
import os

import numpy as np
import pytest

import patchtable_b200 as ptb
from oracle.oracle import mean_dist, recompute_dists
from patchtable_b200 import synth
from tests.conftest import ROOT, srand_all

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_golden.json")))
DESC_TOL = 1e-6        # x sum of |terms| of each projection (float summation error bound)
DIST_RTOL = 1e-5       # NNF_DIST vs float64 recompute
MEAN_DIST_SLACK = 1.01


def _masks():
    spec = importlib.util.spec_from_file_location("gen", os.path.join(ROOT, "patchtable_b200", "csrc", "gen_wh_tables.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    return gen.masks(16)


def exact_descriptor(oracle, img, ndims, nchroma, convert=True, lab=False):
    """float64 descriptor of every full patch, from the oracle's (bit-exact) YUV or Lab image,
    and the sum of |terms| of each projection."""
    from numpy.lib.stride_tricks import sliding_window_view
    conv = oracle.rgb2lab if lab else oracle.rgb2yuv
    yuv = (conv(img) if convert else img).astype(np.float64)
    H, W, _ = yuv.shape
    win = sliding_window_view(yuv, (8, 8), axis=(0, 1))[:H - 7, :W - 7]
    ms = _masks()
    n = ndims - 2 * nchroma
    out = np.zeros((H - 7, W - 7, ndims))
    mag = np.zeros((H - 7, W - 7, ndims))
    for k in range(n):
        M = np.outer(*ms[k])
        planes = range(3) if k < nchroma else [0]
        c0 = 3 * k if k < nchroma else 3 * nchroma + (k - nchroma)
        for j, c in enumerate(planes):
            out[..., c0 + j] = (win[:, :, c] * M).sum(axis=(-1, -2))
            mag[..., c0 + j] = np.abs(win[:, :, c]).sum(axis=(-1, -2))
    return out, mag


@pytest.mark.parametrize("h,w,sw", [(240, 320, ""), (53, 37, "-ndims 8"), (8, 8, "-ndims 7"), (9, 200, "-colorspace rgb"),
                                    (71, 66, "-ndims 4 -nchroma 0"), (130, 90, "-ndims 12 -nchroma 1"),
                                    (90, 120, "-colorspace lab"), (64, 70, "-colorspace lab -ndims 8")])
def test_descriptor_accuracy(gpu, oracle, h, w, sw):
    _, b = synth.pair(h, w, 3)
    p = ptb.PatchTableParams(sw)
    got = ptb.descriptor(p, b).astype(np.float64)
    ex, mag = exact_descriptor(oracle, b, p.ndims, p.nchroma, convert=p.convert_colorspace, lab=p.colorspace == 1)
    orc = oracle.descriptor(p.as_dict(), b)[7:h, 7:w].astype(np.float64)
    tol = DESC_TOL * mag + 1e-30
    assert (np.abs(got - ex) <= tol).all()
    assert (np.abs(got - orc) <= np.abs(orc - ex) + tol).all()


BUILD_CASES = [c for c in GOLDEN["cases"]]


@pytest.mark.parametrize("case", BUILD_CASES, ids=[c["name"] for c in BUILD_CASES])
def test_build_bit_exact_given_descriptors(gpu, oracle, libc, case):
    a, b = synth.pair(case["h"], case["w"], case["seed"])
    p = ptb.PatchTableParams(case["switches"])
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b, wh0=ot.wh0())
    ns, nc = gt.shape()
    assert ns == ot.shape()[0] == case["nslices"]
    assert gt.add_count() == ot.add_count() == case["add_count"]
    for d in range(len(ns)):
        po, pg = ot.partition(d), gt.partition(d)
        for k in po:
            assert np.array_equal(po[k], pg[k]), (d, k)
    tg = gt.table()
    assert np.array_equal(tg, ot.table())
    assert (tg != (1 << 30) - 1).all()
    if p.kcoherence > 0:
        kg, ko = gt.kcoherence(), ot.kcoherence()
        assert np.array_equal(kg[0], ko[0])
        assert np.array_equal(kg[1], ko[1])


DT_CASES = [("-limit 0.5 -nslices 40,9,6,5,4,3,3", 60, 90, 21, False),
            ("-limit 1 -ndims 8", 73, 41, 5, True),
            ("-limit 0.05 -grid_ndims 1", 40, 300, 6, False),
            ("-limit 3 -grid_ndims 2", 50, 60, 7, True)]


@pytest.mark.parametrize("algo", ["downsample", "hybrid", "euclidean"])
@pytest.mark.parametrize("sw,h,w,seed,masked", DT_CASES)
def test_other_distance_transforms(gpu, oracle, libc, algo, sw, h, w, seed, masked):
    """dt_algo downsample / hybrid / euclidean: the filled table equals the oracle's bit for bit,
    including one- and two-dimensional grids and allowed-patch masks (the oracle itself is pinned
    to the reference by the golden digests)."""
    a, b = synth.pair(h, w, seed)
    allowed = None
    if masked:
        rng = np.random.default_rng(seed)
        allowed = (rng.random((h - 7, w - 7)) < 0.7).astype(np.int32)
    p = ptb.PatchTableParams(sw + " -dt_algo " + algo)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b, allowed=allowed)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b, wh0=ot.wh0(), allowed_patches=allowed)
    assert gt.add_count() == ot.add_count()
    tg = gt.table()
    assert np.array_equal(tg, ot.table())
    assert (tg != (1 << 30) - 1).all()
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)


def _flat_bar(h, w, seed, x0, x1):
    """A seeded pair with one constant vertical bar: the bar's patches share one descriptor, so
    their nearest neighbours are each other, most of them within kcoherence_min_dist."""
    a, b = synth.pair(h, w, seed)
    a, b = a.copy(), b.copy()
    a[:, x0:x1] = 0.5
    b[:, x0:x1] = 0.5
    return a, b


@pytest.mark.parametrize("args,sw,knn_min", [((60, 90, 73, 30, 44), "-limit 0.2 -kcoherence 4", 16),
                                             ((70, 80, 74, 20, 60), "-limit 0.2 -kcoherence 6 -kcoherence_min_dist 14", 256),
                                             ((64, 72, 75, 10, 70), "-limit 0.2 -kcoherence 3 -kcoherence_min_dist 12", 128)])
def test_kcoherence_long_neighbour_lists(gpu, oracle, libc, args, sw, knn_min):
    """k-coherence sets whose search needs more than 64 neighbours (the reference doubles knn
    without bound): the set, the table and the query equal the oracle's, which is pinned to the
    reference on the same inputs."""
    a, b = _flat_bar(*args)
    p = ptb.PatchTableParams(sw)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    assert ot.kc_max_knn() >= knn_min
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b, wh0=ot.wh0())
    kg, ko = gt.kcoherence(), ot.kcoherence()
    assert np.array_equal(kg[0], ko[0])
    assert np.array_equal(kg[1], ko[1])
    assert np.array_equal(gt.table(), ot.table())
    check_nnf(oracle, a, b, gt.lookup(a))


@pytest.mark.parametrize("sw,masked", [("-limit 0.5 -kcoherence 3 -kcoherence_step 2 -flann_build_step 2 -flann_reset_step 3", False),
                                       ("-limit 0.5 -kcoherence 3 -kcoherence_step 2 -flann_build_step 2 -flann_reset_step 3", True),
                                       ("-limit 0.5 -kcoherence 2 -flann_reset_step 1", False),
                                       ("-limit 0.5 -kcoherence 2 -flann_reset_step 1", True),
                                       ("-limit 0.5 -kcoherence 2 -kcoherence_step 3 -flann_reset_step 4", True)])
def test_kcoherence_steps_and_segments(gpu, oracle, libc, sw, masked):
    """Sampled train sets (flann_build_step), sampled queries (kcoherence_step) and the knn reset
    segments (flann_reset_step, patchtable.h:2705-2714), with and without an allowed mask: the
    k-coherence set and the table equal the oracle's bit for bit.  The masks leave out the first
    patches of the top row, so the first allowed query opens a segment off the reset columns."""
    a, b = synth.pair(70, 90, 27)
    allowed = None
    if masked:
        rng = np.random.default_rng(27)
        allowed = (rng.random((63, 83)) < 0.8).astype(np.int32)
        allowed[0, :5] = 0
    p = ptb.PatchTableParams(sw)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b, allowed=allowed)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b, wh0=ot.wh0(), allowed_patches=allowed)
    kg, ko = gt.kcoherence(), ot.kcoherence()
    assert np.array_equal(kg[0], ko[0])
    assert np.array_equal(kg[1], ko[1])
    assert np.array_equal(gt.table(), ot.table())
    check_nnf(oracle, a, b, gt.lookup(a))


BRUTE_CASES = [("-limit 0.002", 60, 90, 21, False), ("-limit 0.004 -ndims 8", 43, 71, 5, True),
               ("-limit 0.0005 -grid_ndims 2", 40, 60, 6, False), ("-limit 0.003 -nchroma 0 -ndims 5", 50, 50, 8, True),
               ("-limit 0.01 -grid_ndims 7 -ndims 7", 80, 100, 9, False)]


@pytest.mark.parametrize("sw,h,w,seed,masked", BRUTE_CASES)
def test_brute_distance_transform(gpu, oracle, libc, sw, h, w, seed, masked):
    """dt_algo brute: each cell's nearest patch under the partition's infinity norm equals the
    oracle's bit for bit (the oracle is pinned to the reference directly and by golden digests)."""
    a, b = synth.pair(h, w, seed)
    allowed = None
    if masked:
        rng = np.random.default_rng(seed)
        allowed = (rng.random((h - 7, w - 7)) < 0.7).astype(np.int32)
    p = ptb.PatchTableParams(sw + " -dt_algo brute")
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b, allowed=allowed)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b, wh0=ot.wh0(), allowed_patches=allowed)
    assert np.array_equal(gt.table(), ot.table())
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)


def test_switches_without_effect(gpu, libc):
    """-randomize_dt 1 -populate_nearest 0 are accepted and, as in the reference's build, change
    neither the table nor the query."""
    a, b = synth.pair(70, 90, 12)
    out = []
    for sw in ("-limit 0.5", "-limit 0.5 -randomize_dt 1 -populate_nearest 0"):
        srand_all(libc, 1)
        t = ptb.PatchTable(ptb.PatchTableParams(sw), b)
        out.append((t.table(), t.lookup(a)))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("sw", ["-limit 1 -ntables 3 -coherence_spatial 2", "-speed 3 -ntables 4",
                                "-limit 0.5 -ntables 2 -table_ratio 4 -kcoherence 3"])
def test_multiple_tables(gpu, oracle, libc, sw):
    """ntables > 1: every further table equals the oracle's bit for bit (same rand() stream, limit
    int(limit / table_ratio^i), no k-coherence), and the query tries their entries."""
    a, b = synth.pair(90, 120, 7)
    p = ptb.PatchTableParams(sw)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b, wh0=ot.wh0())
    assert np.array_equal(gt.table(), ot.table())
    for i in range(p.ntables - 1):
        gs, os_ = gt.sub_table(i), ot.sub_table(i)
        assert gs.shape()[0] == os_.shape()[0]
        assert np.array_equal(gs.table(), os_.table()), i
    with pytest.raises(ptb.PatchTableError):
        gt.sub_table(p.ntables - 1)
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * mean_dist(ot.lookup(a))
    # the table step with more tables is never worse than with the first one alone
    q = ptb.PatchTableParams(sw + " -do_prop 0 -kcoherence 0 -prop_iters 1")
    one = ptb.PatchTableParams(sw + " -do_prop 0 -kcoherence 0 -prop_iters 1 -ntables 1")
    srand_all(libc, 1)
    tm = ptb.PatchTable(q, b)
    srand_all(libc, 1)
    t1 = ptb.PatchTable(one, b)
    assert (tm.lookup(a)[..., 2] <= t1.lookup(a)[..., 2]).all()


@pytest.mark.parametrize("spatial", [1, 2])
def test_spatial_search_exact(gpu, oracle, libc, spatial):
    """With one pass and no propagation every patch is independent in the reference too: table
    entry, then the spatial search around it (patchtable.h:3855-3873).  In descriptor mode both
    sides see identical query descriptors, hence identical table entries, and the GPU result
    equals the oracle's bit for bit."""
    a, b = synth.descriptor_pair(70, 90, 8, 23)
    sw = ("-limit 0.5 -kcoherence 0 -do_prop 0 -prop_iters 1 -spatial %d -gpu_prop_passes 1 -is_descriptor 1"
          % spatial)
    p = ptb.PatchTableParams(sw)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    assert np.array_equal(gt.table(), ot.table())
    assert np.array_equal(gt.lookup(a), ot.lookup(a))


@pytest.mark.parametrize("speed", list(range(10)))
def test_every_speed_preset(gpu, oracle, libc, speed):
    """Every -speed preset (patchtable.cpp:138-149: random and spatial search, k-coherence up to 20,
    query_step up to 10) runs, with a mean distance at most 1 % above the oracle's."""
    a, b = synth.pair(150, 200, 30 + speed)
    p = ptb.PatchTableParams("-speed %d -limit 2" % speed)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 5)
    mo = mean_dist(ot.lookup(a))
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * mo, (mean_dist(ann), mo)


def test_init_random(gpu, oracle, libc):
    """init_random (patchtable.h:3522-3537) starts every patch from a random match with its exact
    distance; the table step and propagation then refine it like the reference's."""
    a, b = synth.pair(120, 150, 25)
    p = ptb.PatchTableParams("-limit 2 -init_random 1")
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)
    srand_all(libc, 2)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * mean_dist(ot.lookup(a))
    # without table lookup or propagation the field is the random start itself: exact distances
    q = ptb.PatchTableParams("-limit 2 -init_random 1 -do_table_lookup 0 -do_prop 0 -kcoherence 0")
    srand_all(libc, 1)
    t0 = ptb.PatchTable(q, b)
    start = t0.lookup(a)
    check_nnf(oracle, a, b, start)
    assert np.array_equal(start, t0.lookup(a))          # the hashed start does not depend on rand()
    assert mean_dist(start) > 2 * mean_dist(ann)


def check_nnf(oracle, a, b, ann, sample=4000):
    eh, ew = a.shape[0] - 7, a.shape[1] - 7
    beh, bew = b.shape[0] - 7, b.shape[1] - 7
    assert ann.shape == (eh, ew, 3)
    bx, by = ann[..., 0], ann[..., 1]
    assert (bx == np.round(bx)).all() and (by == np.round(by)).all()
    assert (bx >= 0).all() and (bx < bew).all() and (by >= 0).all() and (by < beh).all()
    rd = recompute_dists(a, b, ann)
    rel = np.abs(ann[..., 2] - rd) / np.maximum(rd, 1e-12)
    assert rel.max() <= DIST_RTOL
    rng = np.random.default_rng(0)
    ys = rng.integers(0, eh, sample)
    xs = rng.integers(0, ew, sample)
    for y, x in zip(ys, xs):
        d = oracle.patch_dist(a, x, y, b, int(bx[y, x]), int(by[y, x]))
        assert np.float32(ann[y, x, 2]) == np.float32(d)


@pytest.mark.parametrize("seed,sw", [(1, ""), (2, ""), (3, "-coherence_spatial 4"), (1, "-coherence_spatial 4"),
                                     (4, "-kcoherence 4 -prop_iters 3"), (5, "-speed 6"), (6, "-kcoherence_iter 1"),
                                     (7, "-kcoherence 4 -kcoherence_iter 0"), (8, "-kcoherence_iter 2 -prop_iters 3")])
def test_nnf_quality_and_distances(gpu, oracle, libc, seed, sw):
    """Exact distances and the mean within 1% of the oracle's; -kcoherence_iter n restricts
    k-coherence to the passes of sweep n (patchtable.h:3612), and repeated lookups are identical."""
    a, b = synth.pair(240, 320, seed)
    p = ptb.PatchTableParams(sw + " -limit 10")
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    mo = mean_dist(ot.lookup(a))
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)
    mg = mean_dist(ann)
    assert mg <= MEAN_DIST_SLACK * mo, (mg, mo)
    assert np.array_equal(ann, gt.lookup(a))


@pytest.mark.parametrize("sw", ["", "-coherence_spatial 4 -kcoherence 4", "-speed 6"])
def test_kcoherence_cap(gpu, oracle, libc, sw):
    """gpu_kc_max: a cap at or above kcoherence changes nothing; -1 is exactly the query without
    the k-coherence step (kcoherence_iter past every sweep); 1 tries only each list's first
    neighbour.  Distances stay exact, the table is untouched."""
    a, b = synth.pair(200, 260, 31)
    p = ptb.PatchTableParams(sw + " -limit 10")
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    table = gt.table()
    full = gt.lookup(a)
    p.gpu_kc_max = p.kcoherence
    assert np.array_equal(gt.lookup(a), full)
    p.gpu_kc_max = -1
    none = gt.lookup(a)
    check_nnf(oracle, a, b, none, sample=500)
    p.gpu_kc_max = 0
    p.kcoherence_iter = 99
    assert np.array_equal(gt.lookup(a), none)
    p.kcoherence_iter = -1
    p.gpu_kc_max = 1
    one = gt.lookup(a)
    check_nnf(oracle, a, b, one, sample=500)
    assert np.array_equal(gt.table(), table)


def test_query_of_another_size_and_reuse(gpu, oracle, libc):
    _, b = synth.pair(150, 170, 7)
    p = ptb.PatchTableParams("-limit 2")
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    for (h, w, s) in [(90, 260, 8), (150, 170, 9), (33, 41, 10), (90, 260, 8)]:
        a = synth.image_a(h, w, s)
        ann1 = gt.lookup(a)
        ann2 = gt.lookup(a)
        assert np.array_equal(ann1, ann2)
        check_nnf(oracle, a, b, ann1, sample=500)


def test_device_lookup_matches_host(gpu, libc):
    import torch
    a, b = synth.pair(120, 160, 12)
    p = ptb.PatchTableParams("-limit 2")
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    host = gt.lookup(a)
    da = torch.from_numpy(a).to(gpu)
    dann = torch.empty((113, 153, 3), dtype=torch.float64, device=gpu)
    gt.lookup_device(da.data_ptr(), 120, 160, dann.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(dann.cpu().numpy(), host)


def test_small_and_degenerate_images(gpu, libc):
    srand_all(libc, 1)
    for (h, w) in [(8, 8), (9, 13), (15, 200), (200, 9)]:
        _, b = synth.pair(h, w, 31)
        a = synth.image_a(h + 3, w + 5, 32)
        p = ptb.PatchTableParams("-limit 0.01 -kcoherence 0")
        gt = ptb.PatchTable(p, b)
        ann = gt.lookup(a)
        assert ann.shape == (h + 3 - 7, w + 5 - 7, 3)
        assert (ann[..., 0] < w - 7).all() and (ann[..., 1] < h - 7).all()
    with pytest.raises(ptb.PatchTableError):
        ptb.PatchTable(ptb.PatchTableParams("-limit 0.01"), synth.pair(8, 8, 1)[1])   # k-coherence needs neighbours


@pytest.mark.parametrize("h,w", [(12, 65535), (16383, 9)])
def test_maximum_extents(gpu, oracle, libc, h, w):
    """The largest sides of b a packed position XY_TO_INT holds (x < 2^16; y < 2^14 keeps every
    position below TABLE_UNUSED): the table builds and the query returns exact distances; one
    pixel more along that side is rejected for the table.  Query positions are never packed, so a
    query one pixel larger is answered like any other."""
    a, b = synth.pair(h, w, 61)
    srand_all(libc, 1)
    t = ptb.PatchTable(ptb.PatchTableParams("-limit 0.05 -kcoherence 2"), b)
    check_nnf(oracle, a, b, t.lookup(a))
    hh, ww = (h, w + 1) if w == 65535 else (h + 1, w)
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTable(ptb.PatchTableParams("-limit 0.05"), np.zeros((hh, ww, 3), np.float32))
    assert e.value.status == 1
    a2 = synth.image_a(hh, ww, 62)
    check_nnf(oracle, a2, b, t.lookup(a2))


def test_constant_image(gpu, libc):
    """Zero range in every dimension (get_bin divides 0 by 0) must still build and match."""
    b = np.full((40, 50, 3), 0.25, np.float32)
    a = np.full((30, 30, 3), 0.5, np.float32)
    srand_all(libc, 1)
    gt = ptb.PatchTable(ptb.PatchTableParams("-limit 0.1"), b)
    ann = gt.lookup(a)
    assert np.allclose(ann[..., 2], 64 * 3 * 0.0625)


@pytest.mark.parametrize("sw", ["-incoherence 1", "-dt_algo raster", "-dt_algo kdtree", "-ntables 17",
                                "-dim_algo pca -pca_mean 1"])
def test_unsupported_options_fail_loudly(gpu, sw):
    _, b = synth.pair(40, 40, 1)
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTable(ptb.PatchTableParams(sw), b)
    assert e.value.status == 5


def test_full_size_1920x1080(gpu, oracle, libc):
    """The headline workload, checked through size-independent properties and the reference's
    mean distance recorded in the golden file."""
    g = GOLDEN["c2"]
    a, b = synth.pair(g["h"], g["w"], g["seed"])
    srand_all(libc, 1)
    gt = ptb.PatchTable(ptb.PatchTableParams(g["switches"]), b)
    tab = gt.table()
    assert (tab != (1 << 30) - 1).all()
    assert ((tab & 0xFFFF) >= 7).all() and ((tab & 0xFFFF) < g["w"]).all()
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann, sample=2000)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * g["mean_dist"]
