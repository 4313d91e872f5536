"""Table files in the reference's format (PatchTableFixedN::save/load, patchtable.h:1574-1622):
our files load into the reference (oracle/_ref) and the reference's files load into this
library, with bit-identical tables and partitions, and a saved and reloaded table answers
queries exactly like the original."""
import numpy as np
import pytest

import patchtable_b200 as ptb
from patchtable_b200 import synth

from tests.test_gpu_parity import check_nnf

pytestmark = pytest.mark.gpu
SW = "-speed 3 -coherence_spatial 4 -limit 2"


def _same_structure(ours, ref_or_ours):
    ns, nc = ours.shape()
    ns2, nc2 = ref_or_ours.shape()
    assert ns == ns2 and nc == nc2
    assert np.array_equal(ours.table(), ref_or_ours.table())
    for d in range(len(ns)):
        a, b = ours.partition(d), ref_or_ours.partition(d)
        for k in ("centers", "lsizes", "rsizes", "to_bin"):
            assert np.array_equal(a[k], b[k]), (d, k)
        for k in ("min", "max", "range"):
            assert a[k] == b[k], (d, k)


def test_roundtrip_answers_like_the_original(gpu, libc, tmp_path):
    a, b = synth.pair(120, 160, 41)
    p = ptb.PatchTableParams(SW)
    libc.srand(1)
    t = ptb.PatchTable(p, b)
    f = tmp_path / "t.ptbl"
    t.save(f)
    t2 = ptb.PatchTable.load(ptb.PatchTableParams(SW), f)
    assert t2.shape_b == (120, 160, 3)
    _same_structure(t, t2)
    assert np.array_equal(t.kcoherence()[0], t2.kcoherence()[0])
    assert np.array_equal(t.lookup(a), t2.lookup(a))


def test_switches_save_and_load(gpu, libc, tmp_path):
    a, b = synth.pair(100, 130, 42)
    f = tmp_path / "s.ptbl"
    libc.srand(1)
    t = ptb.PatchTable(ptb.PatchTableParams(SW + " -save %s" % f), b)
    assert f.exists()
    t2 = ptb.PatchTable(ptb.PatchTableParams(SW + " -load %s" % f), b)
    _same_structure(t, t2)


def test_reference_loads_our_file(gpu, libc, reference, tmp_path):
    a, b = synth.pair(110, 140, 43)
    libc.srand(1)
    t = ptb.PatchTable(ptb.PatchTableParams(SW), b)
    f = tmp_path / "ours.ptbl"
    t.save(f)
    rt = reference.build(SW + " -load %s" % f, b)
    _same_structure(t, rt)


def test_we_load_the_reference_file(gpu, oracle, libc, reference, tmp_path):
    a, b = synth.pair(110, 140, 44)
    f = tmp_path / "ref.ptbl"
    reference.srand(1)
    rt = reference.build(SW + " -save %s" % f, b)
    t = ptb.PatchTable.load(ptb.PatchTableParams(SW), f)
    _same_structure(t, rt)
    check_nnf(oracle, a, b, t.lookup(a))


def test_bad_files_fail_cleanly(gpu, libc, tmp_path):
    f = tmp_path / "junk"
    f.write_bytes(b"not a table")
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTable.load(ptb.PatchTableParams(SW), f)
    assert e.value.status == 6
    a, b = synth.pair(60, 70, 45)
    libc.srand(1)
    g = tmp_path / "g.ptbl"
    ptb.PatchTable(ptb.PatchTableParams(SW), b).save(g)
    data = g.read_bytes()
    (tmp_path / "cut").write_bytes(data[: len(data) // 2])
    with pytest.raises(ptb.PatchTableError):
        ptb.PatchTable.load(ptb.PatchTableParams(SW), tmp_path / "cut")
    with pytest.raises(ptb.PatchTableError) as e:
        ptb.PatchTable.load(ptb.PatchTableParams(SW + " -ndims 8"), g)
    assert e.value.status == 1
