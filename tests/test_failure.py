"""Failure paths without a GPU fault (the reference prints and exits on every error,
solver/util.h:31-32; this library returns a status and stays usable).

* A bounded device wait that runs out: with the spin limit at 0, the first grid-barrier wait of
  the cooperative table build gives up at once; every block leaves, the build returns PT_TIMEOUT,
  and the next build on the same device succeeds with the same table as before.
* Out of device memory: with the library's allocation cap below what a build or a lookup needs,
  the call returns PT_OOM, holds no memory afterwards, and works again once the cap is lifted.
"""
import numpy as np
import pytest

import patchtable_b200 as ptb
from patchtable_b200 import synth
from tests.conftest import srand_all

PT_OOM, PT_TIMEOUT = 2, 4


def test_limits_are_process_wide_settings():
    old = ptb.set_spin_limit(123)
    try:
        assert ptb.set_spin_limit(456) == 123
    finally:
        ptb.set_spin_limit(-1)
    assert ptb.set_spin_limit(-1) == 1 << 24
    ptb.set_spin_limit(old)
    prev = ptb.set_device_alloc_limit(1 << 20)
    try:
        assert ptb.set_device_alloc_limit(-1) == 1 << 20
    finally:
        ptb.set_device_alloc_limit(prev)


@pytest.mark.gpu
def test_build_barrier_wait_times_out_and_device_stays_usable(gpu, libc):
    _, b = synth.pair(120, 160, 51)
    p = ptb.PatchTableParams("-limit 1")
    srand_all(libc, 1)
    good = ptb.PatchTable(p, b).table()
    old = ptb.set_spin_limit(0)
    try:
        srand_all(libc, 1)
        with pytest.raises(ptb.PatchTableError) as e:
            ptb.PatchTable(p, b)
        assert e.value.status == PT_TIMEOUT
        assert "gave up" in str(e.value)
    finally:
        ptb.set_spin_limit(old)
    srand_all(libc, 1)
    assert np.array_equal(ptb.PatchTable(p, b).table(), good)


@pytest.mark.gpu
def test_out_of_memory_is_reported_and_recovered(gpu, libc):
    a, b = synth.pair(150, 200, 52)
    p = ptb.PatchTableParams("-limit 1")
    base = ptb.device_bytes_in_use()
    old = ptb.set_device_alloc_limit(base + (1 << 20))
    try:
        srand_all(libc, 1)
        with pytest.raises(ptb.PatchTableError) as e:
            ptb.PatchTable(p, b)
        assert e.value.status == PT_OOM
    finally:
        ptb.set_device_alloc_limit(old)
    assert ptb.device_bytes_in_use() == base
    srand_all(libc, 1)
    t = ptb.PatchTable(p, b)
    held = ptb.device_bytes_in_use()
    # a lookup needs its query buffers: refused under a cap at the table's own footprint
    old = ptb.set_device_alloc_limit(held)
    try:
        with pytest.raises(ptb.PatchTableError) as e:
            t.lookup(a)
        assert e.value.status == PT_OOM
    finally:
        ptb.set_device_alloc_limit(old)
    ann = t.lookup(a)
    assert ann.shape == (143, 193, 3) and np.isfinite(ann).all()
    t.close()
    assert ptb.device_bytes_in_use() == base
