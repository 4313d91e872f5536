"""Zero-allocation query (pt_table_lookup_device_noalloc).

Callers that may not allocate device memory while querying -- a frame loop with a fixed latency
budget, where cudaMalloc/cudaFree would synchronise the device, or an application whose own
allocator owns the GPU's memory -- use this entry point; it takes every intermediate buffer from
one static device array.  It must return exactly what pt_table_lookup_device returns, call after
call, although all calls share (and overwrite) that array.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

import patchtable_b200 as ptb
from patchtable_b200 import synth

pytestmark = pytest.mark.gpu


def _fn():
    f = ptb.lib().pt_table_lookup_device_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("sw", ["-limit 2", "-limit 2 -prop_iters 0", "-limit 2 -do_prop 0", "-limit 2 -gpu_tile 128",
                                "-limit 2 -kcoherence_iter 1 -gpu_tile 64", "-limit 2 -gpu_kc_max -1",
                                "-limit 2 -gpu_kc_max 1 -gpu_prop_passes 1"])
def test_noalloc_lookup_matches_device_lookup_on_consecutive_calls(sw):
    import torch
    assert torch.cuda.is_available()
    noalloc = _fn()
    C.CDLL(None).srand(1)
    _, b = synth.pair(200, 260, 41)
    table = ptb.PatchTable(ptb.PatchTableParams(sw), b)
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row on the same image, then a call on an image of another size
    for (h, w, seed) in [(300, 400, 42), (300, 400, 42), (257, 509, 43)]:
        a = synth.image_a(h, w, seed)
        da = torch.from_numpy(a).cuda()
        expect = torch.empty((h - 7, w - 7, 3), dtype=torch.float64, device="cuda")
        got = torch.full((h - 7, w - 7, 3), float("nan"), dtype=torch.float64, device="cuda")
        table.lookup_device(da.data_ptr(), h, w, expect.data_ptr(), stream)
        st = noalloc(table._h, da.data_ptr(), h, w, got.data_ptr(), stream)
        assert st == 0, ptb.lib().pt_last_error()
        torch.cuda.synchronize()
        assert torch.equal(expect, got)
    table.close()


def test_noalloc_lookup_allocates_no_device_memory():
    """After a first call (which may load the kernels), further calls leave the device's free
    memory unchanged: nothing is allocated, not even temporarily for the call's duration."""
    import torch
    noalloc = _fn()
    C.CDLL(None).srand(1)
    _, b = synth.pair(150, 190, 45)
    table = ptb.PatchTable(ptb.PatchTableParams("-limit 1"), b)
    stream = torch.cuda.current_stream().cuda_stream
    h, w = 240, 320
    da = torch.from_numpy(synth.image_a(h, w, 46)).cuda()
    out = torch.empty((h - 7, w - 7, 3), dtype=torch.float64, device="cuda")
    assert noalloc(table._h, da.data_ptr(), h, w, out.data_ptr(), stream) == 0, ptb.lib().pt_last_error()
    torch.cuda.synchronize()
    first = out.clone()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert noalloc(table._h, da.data_ptr(), h, w, out.data_ptr(), stream) == 0, ptb.lib().pt_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.equal(first, out)
    table.close()


def test_noalloc_rejects_images_over_the_limit():
    import torch
    noalloc = _fn()
    C.CDLL(None).srand(1)
    _, b = synth.pair(64, 64, 44)
    table = ptb.PatchTable(ptb.PatchTableParams("-limit 0.1"), b)
    da = torch.zeros((600, 600, 3), dtype=torch.float32, device="cuda")
    out = torch.zeros((593, 593, 3), dtype=torch.float64, device="cuda")
    st = noalloc(table._h, da.data_ptr(), 600, 600, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 1
    assert b"at most" in ptb.lib().pt_last_error()
