"""The C ABI library loads without a GPU, exports every declared entry point, and rejects bad
arguments with status codes (no GPU work is issued by these checks)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import patchtable_b200 as ptb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h") or fn == "patchtable_compat.h":
            continue
        txt = open(os.path.join(ROOT, "include", fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    lib = ptb.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_slot():
    assert b"sm_100a" in ptb.lib().pt_version()
    assert isinstance(ptb.lib().pt_last_error(), bytes)


def test_bad_arguments_are_rejected_before_device_work():
    p = ptb.PatchTableParams()
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTable(p, np.zeros((7, 30, 3), np.float32))
    assert e.value.status == 1
    with pytest.raises(ptb.PatchTableError):
        ptb.PatchTable(p, np.zeros((30, 30), np.float32))
    bad = ptb.PatchTableParams("-patch_w 7")
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTable(bad, np.zeros((30, 30, 3), np.float32))
    assert e.value.status == 5
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTableParams("-speed 12")
    assert e.value.status == 1
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTableParams("-dt_algo nosuch")
    assert e.value.status == 1
