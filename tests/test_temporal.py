"""Temporal lookups (PatchTable::lookup with ann_prev / coherence_temporal_sv,
patchtable.h:3548-3585, 4178-4193): the previous frame's NNF seeds the field, its distances are
recomputed and scaled by 1/(1+coherence_temporal) (or the per-patch scale), and a patch that keeps
its previous match gets the unscaled distance back."""
import numpy as np
import pytest

import patchtable_b200 as ptb
from oracle.oracle import mean_dist
from patchtable_b200 import synth

from tests.test_gpu_parity import MEAN_DIST_SLACK, check_nnf

pytestmark = pytest.mark.gpu
SW = "-speed 3 -coherence_spatial 4 -limit 2"


def test_previous_field_never_gets_worse(gpu, oracle, libc):
    a, b = synth.pair(120, 160, 51)
    p = ptb.PatchTableParams(SW + " -coherence_temporal 0")
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    p.gpu_prop_passes = 1
    prev = t.lookup(a)
    again = t.lookup(a, ann_prev=prev)
    check_nnf(oracle, a, b, again)
    assert np.all(again[..., 2] <= prev[..., 2])


@pytest.mark.parametrize("recalc", [1, 0])
def test_temporal_matches_oracle_quality(gpu, oracle, libc, recalc):
    a0, b = synth.pair(150, 200, 52)
    a1 = synth.crop(synth.warp(a0, 53), 150, 200, 53)
    sw = SW + " -coherence_temporal 2 -recalc_dist_temporal %d" % recalc
    p = ptb.PatchTableParams(sw)
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    prev = t.lookup(a0)
    ours = t.lookup(a1, ann_prev=prev)
    libc.srand(1)
    ot = oracle.build(p.as_dict(), b)
    ref = ot.lookup(a1, ann_prev=prev)
    if recalc:
        check_nnf(oracle, a1, b, ours)
    kept = (ours[..., 0] == prev[..., 0]) & (ours[..., 1] == prev[..., 1])
    assert kept.mean() > 0.05
    assert mean_dist(ours) <= MEAN_DIST_SLACK * mean_dist(ref), (mean_dist(ours), mean_dist(ref))


def test_per_patch_scale_and_sanitize(gpu, oracle, libc):
    a, b = synth.pair(100, 130, 54)
    p = ptb.PatchTableParams(SW + " -coherence_temporal 1")
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    prev = t.lookup(a)
    rng = np.random.default_rng(0)
    sv = rng.uniform(0.3, 1.0, prev.shape[:2]).astype(np.float32)
    out = t.lookup(a, ann_prev=prev, coherence_temporal_sv=sv)
    assert np.all(out[..., 0] < b.shape[1] - 7) and np.all(out[..., 1] < b.shape[0] - 7)
    bad = prev.copy()
    bad[0, 0, 0] = 10 * b.shape[1]
    check_nnf(oracle, a, b, t.lookup(a, ann_prev=bad))           # clamped (sanitize_input 1)
    p.sanitize_input = 0
    with pytest.raises(ptb.PatchTableError):
        t.lookup(a, ann_prev=bad)
    with pytest.raises(ptb.PatchTableError):
        t.lookup(a, ann_prev=prev[:-1])


def test_temporal_with_multiple_tables(gpu, libc):
    """ann_prev seeding composes with further tables: the seeded lookup never ends worse than its
    seed and its distances are exact."""
    a, b = synth.pair(120, 150, 88)
    p = ptb.PatchTableParams("-limit 2 -ntables 3 -coherence_temporal 0")
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    first = t.lookup(a)
    again = t.lookup(a, ann_prev=first)
    assert (again[..., 2] <= first[..., 2]).all()
