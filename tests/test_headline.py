"""The 1920x1080 workload that bench.py measures, pinned to the reference.

* CPU: the restated descriptor of the table image has the digest of the reference's wh0 at this
  size (tests/golden/oracle_golden.json, entry c2, written by tests/golden/make_golden.py from the
  reference sources compiled in place).
* GPU: given that descriptor, the GPU build's partition, table after the DT and k-coherence set
  have the reference's digests, bit for bit.
* GPU: every query schedule the bench may time (its SCHEDULES, at the CTA width it usually picks,
  with and without the k-coherence step) returns exact, in-bounds distances (NNF_DIST bit-exact with patch_dist_exact, within 1e-5 of a
  float64 recompute), the same field through the device entry point and the host lookup, and a
  mean NNF distance at most 1% above the reference's.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import patchtable_b200 as ptb
from bench import SCHEDULES
from oracle.oracle import mean_dist
from patchtable_b200 import synth
from tests.conftest import ROOT, srand_all
from tests.test_gpu_parity import MEAN_DIST_SLACK, check_nnf

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_golden.json")))["c2"]


def digest(arr):
    return hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def c2_pair():
    return synth.pair(GOLDEN["h"], GOLDEN["w"], GOLDEN["seed"])


@pytest.fixture(scope="module")
def c2_wh0(oracle, c2_pair):
    return oracle.descriptor(ptb.PatchTableParams(GOLDEN["switches"]).as_dict(), c2_pair[1])


def test_c2_descriptor_matches_reference(c2_wh0):
    assert digest(c2_wh0) == GOLDEN["wh0"]


@pytest.mark.gpu
def test_c2_build_bit_exact_given_reference_descriptor(gpu, libc, c2_pair, c2_wh0):
    p = ptb.PatchTableParams(GOLDEN["switches"])
    srand_all(libc, 1)
    t = ptb.PatchTable(p, c2_pair[1], wh0=c2_wh0)
    ns, _ = t.shape()
    assert list(ns) == GOLDEN["nslices"]
    assert t.add_count() == GOLDEN["add_count"]
    parts = [t.partition(d) for d in range(len(ns))]
    flat = np.concatenate([np.concatenate([q["centers"], q["lsizes"], q["rsizes"], q["to_bin"].view(np.float32),
                                           [q["min"], q["max"], q["range"]]]) for q in parts])
    assert digest(flat) == GOLDEN["partition"]
    assert digest(t.table()) == GOLDEN["table"]
    kp, kd = t.kcoherence()
    assert digest(kp) == GOLDEN["kcoh_pos"]
    assert digest(kd) == GOLDEN["kcoh_dist"]
    t.close()


@pytest.fixture(scope="module")
def c2_table(gpu, libc, c2_pair):
    srand_all(libc, 1)
    t = ptb.PatchTable(ptb.PatchTableParams(GOLDEN["switches"]), c2_pair[1])
    yield t
    t.close()


@pytest.mark.gpu
@pytest.mark.parametrize("sched", SCHEDULES, ids=[ptb.schedule_name(s) for s in SCHEDULES])
def test_benchmarked_schedules(gpu, oracle, c2_pair, c2_table, sched):
    import torch
    a, b = c2_pair
    H, W = a.shape[:2]
    p = c2_table.params
    p.set_schedule(sched)
    p.gpu_tile = 64
    try:
        host = c2_table.lookup(a)
        da = torch.from_numpy(a).to(gpu)
        dann = torch.empty((H - 7, W - 7, 3), dtype=torch.float64, device=gpu)
        c2_table.lookup_device(da.data_ptr(), H, W, dann.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(dann.cpu().numpy(), host)
        check_nnf(oracle, a, b, host, sample=1500)
        assert mean_dist(host) <= MEAN_DIST_SLACK * GOLDEN["mean_dist"], (mean_dist(host), GOLDEN["mean_dist"])
    finally:
        p.set_schedule((0, 0, 0))
        p.gpu_tile = 0
