"""-dim_algo pca: the patch-PCA descriptor (patchtable/patch_pca.h) on the GPU.

The reference fits cv::PCA on pca_samples random patches (consuming rand()) and projects every
patch onto the leading ndims eigenvectors; its patch vectors hold floats dx + c of each patch row
(the row pointer is indexed by dx floats).  OpenCV is not available: oracle/pca_jacobi.h restates
the published PCA (sample mean, covariance, Jacobi eigenvectors ordered by eigenvalue, largest
entry positive) and stands in for cv::PCA inside the reference build, so the reference's own
sampling and projection run and pin the oracle by digest (tests/golden, pca_* cases).  The GPU
path must agree with the oracle: descriptors to float rounding of the independently computed
bases, tables bit-exact given the oracle's descriptors, NNF distances exact and mean distance
within 1 %."""
import ctypes

import numpy as np
import pytest

import patchtable_b200 as ptb
from oracle.oracle import mean_dist
from patchtable_b200 import synth

from tests.conftest import srand_all
from tests.test_gpu_parity import MEAN_DIST_SLACK, check_nnf

pytestmark = pytest.mark.gpu

CASES = [("-dim_algo pca -limit 1", 120, 160, 11), ("-dim_algo pca -ndims 8 -kcoherence 2 -limit 2", 100, 130, 12),
         ("-dim_algo pca -ndims 4 -pca_subtract_mean 0 -pca_samples 300 -limit 0.5", 90, 70, 13),
         ("-dim_algo pca -ndims 12 -colorspace rgb -limit 3", 80, 110, 14),
         ("-dim_algo pca -colorspace lab -limit 1", 90, 120, 15)]


@pytest.mark.parametrize("sw,h,w,seed", CASES)
def test_pca_descriptor_and_table(gpu, oracle, libc, sw, h, w, seed):
    a, b = synth.pair(h, w, seed)
    p = ptb.PatchTableParams(sw)
    srand_all(libc, 1)
    ot = oracle.build(p.as_dict(), b)
    after_oracle = libc.rand()
    srand_all(libc, 1)
    gt = ptb.PatchTable(p, b)
    assert libc.rand() == after_oracle              # same rand() draws: PCA samples, then populate
    want = ot.wh0()[7:h, 7:w]
    got = gt.descriptor()
    scale = np.abs(want).max(axis=(0, 1))
    assert (np.abs(got - want) <= 1e-5 * scale + 1e-7).all(), np.abs(got - want).max()
    # the table and k-coherence set, bit-exact from the oracle's descriptors
    srand_all(libc, 1)
    gw = ptb.PatchTable(p, b, wh0=ot.wh0())
    assert gw.shape()[0] == ot.shape()[0]
    assert np.array_equal(gw.table(), ot.table())
    if p.kcoherence > 0:
        kg, ko = gw.kcoherence(), ot.kcoherence()
        assert np.array_equal(kg[0], ko[0]) and np.array_equal(kg[1], ko[1])
    ann = gt.lookup(a)
    check_nnf(oracle, a, b, ann)
    assert mean_dist(ann) <= MEAN_DIST_SLACK * mean_dist(ot.lookup(a))


def test_pca_unsupported_combinations(gpu, tmp_path):
    _, b = synth.pair(40, 40, 1)
    for sw in ("-dim_algo pca -pca_mean 1", "-dim_algo pca -is_descriptor 1"):
        with pytest.raises(ptb.PatchTableError) as e:
            ptb.PatchTable(ptb.PatchTableParams(sw), b if "is_descriptor" not in sw else np.zeros((20, 20, 6), np.float32))
        assert e.value.status == 5
    t = ptb.PatchTable(ptb.PatchTableParams("-dim_algo pca -limit 0.1"), b)
    with pytest.raises(ptb.PatchTableError) as e:
        t.save(str(tmp_path / "pca.bin"))
    assert e.value.status == 5
