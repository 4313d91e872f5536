"""The C++ compatibility header compiles a reference-style caller (CPU), and that caller
produces the same NNF as the Python binding (GPU)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from patchtable_b200 import synth
from tests.conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "compat_example.cpp")
LIBDIR = os.path.join(ROOT, "patchtable_b200")


def build_example(tmp_path):
    exe = str(tmp_path / "compat_example")
    subprocess.run(["g++", "-std=c++11", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-lpatchtable_b200", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def test_compat_header_compiles_and_links(tmp_path):
    assert os.path.exists(build_example(tmp_path))


@pytest.mark.gpu
def test_compat_caller_matches_python_binding(tmp_path):
    import patchtable_b200 as ptb
    exe = build_example(tmp_path)
    a, b = synth.pair(90, 120, 17)
    a.tofile(str(tmp_path / "a.raw"))
    b.tofile(str(tmp_path / "b.raw"))
    out = tmp_path / "ann.raw"
    r = subprocess.run([exe, "90", "120", str(tmp_path / "a.raw"), str(tmp_path / "b.raw"), str(out), "patchtable",
                        "-limit", "1", "-coherence_spatial", "2"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "mean_dist:" in r.stdout
    ann_cpp = np.fromfile(str(out), dtype=np.float64).reshape(83, 113, 3)
    ctypes.CDLL(None).srand(1)      # the C++ process started from the default rand() state (seed 1)
    t = ptb.PatchTable(ptb.PatchTableParams("-limit 1 -coherence_spatial 2"), b)
    assert np.array_equal(t.lookup(a), ann_cpp)
