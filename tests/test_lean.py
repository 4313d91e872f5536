"""The specialised query kernels (a choose with only the table step, a pull with one neighbour
candidate) against the general kernels they replace: every lookup path -- device, host (banded),
batch and zero-allocation -- gives the same NNF bit for bit with the variants on and off, for
schedules that use one, both or neither of them, with and without an allowed mask."""
import ctypes as C

import numpy as np
import pytest

import patchtable_b200 as ptb
from patchtable_b200 import synth

from tests.test_gpu_parity import check_nnf

pytestmark = pytest.mark.gpu

SCHEDULES = [(1, 2, 1, -1), (2, 2, 1, -1), (1, 2, 1), (1, 2, 2, -1), (2, 1, 1)]


def _lookups(t, a, queries):
    import torch
    h, w = a.shape[:2]
    st = torch.cuda.current_stream().cuda_stream
    da = torch.from_numpy(a).cuda()
    dann = torch.empty((h - 7, w - 7, 3), dtype=torch.float64, device="cuda")
    t.lookup_device(da.data_ptr(), h, w, dann.data_ptr(), st)
    torch.cuda.synchronize()
    out = {"device": dann.cpu().numpy(), "host": t.lookup(a)}
    out["batch"] = t.lookup_batch(queries)
    noalloc = ptb.lib().pt_table_lookup_device_noalloc
    noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    dann2 = torch.empty_like(dann)
    assert noalloc(t._h, C.c_void_p(da.data_ptr()), h, w, C.c_void_p(dann2.data_ptr()), C.c_void_p(st)) == 0
    torch.cuda.synchronize()
    out["noalloc"] = dann2.cpu().numpy()
    return out


@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("sched", SCHEDULES, ids=[ptb.schedule_name(s) for s in SCHEDULES])
def test_lean_kernels_equal_general(gpu, oracle, libc, sched, masked):
    a, b = synth.pair(180, 240, 77)
    allowed = None
    if masked:
        rng = np.random.default_rng(77)
        allowed = (rng.random((173, 233)) < 0.75).astype(np.int32)
    p = ptb.PatchTableParams("-speed 3 -coherence_spatial 4 -limit 2")
    libc.srand(1)
    t = ptb.PatchTable(p, b, allowed_patches=allowed)
    p.set_schedule(sched)
    queries = [a, synth.pair(70, 300, 78)[0], synth.pair(150, 90, 79)[0]]
    prev = ptb.set_lean_kernels(False)
    try:
        general = _lookups(t, a, queries)
        ptb.set_lean_kernels(True)
        lean = _lookups(t, a, queries)
    finally:
        ptb.set_lean_kernels(prev)
    for k in ("device", "host", "noalloc"):
        assert np.array_equal(general[k], lean[k]), k
        assert np.array_equal(lean[k], lean["device"]), k
    for g, l in zip(general["batch"], lean["batch"]):
        assert np.array_equal(g, l)
    assert np.array_equal(lean["batch"][0], lean["device"])
    check_nnf(oracle, a, b, lean["device"], sample=300)
    if masked:
        ann = lean["device"]
        assert (allowed[ann[..., 1].astype(int), ann[..., 0].astype(int)] == 1).all()
    t.close()
