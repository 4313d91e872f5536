"""Parameter defaults, speed presets and switch parsing match the reference's own parser
(PatchTableParams, patchtable/patchtable.cpp:26-373), field by field."""
import pytest

import patchtable_b200 as ptb
from oracle.oracle import PARAM_FIELDS

SWITCHES = [""] + ["-speed %d" % i for i in range(10)] + [
    "-speed 3 -coherence_spatial 4",
    "-limit 1 -kcoherence 5 -prop_iters 3",
    "-ndims 8 -nchroma 1 -limit 0.5",
    "-speed 5 -limit 2 -dt_iters 3 -query_step 2",
    "-nslices 10,10,10,5,5,5",
    "-grid_ndims 4 -triangle_factor 3.5 -kcoherence_min_dist 3",
    "-colorspace rgb -populate_random 0 -run_dt 0",
    "-flann_reset_step 7 -kcoherence_step 2 -partition_step 3",
]


@pytest.mark.parametrize("sw", SWITCHES)
def test_params_match_reference(reference, sw):
    ref = reference.params(sw)
    ours = ptb.PatchTableParams(sw).as_dict()
    for f in PARAM_FIELDS:
        assert ours[f] == pytest.approx(ref[f]), (sw, f, ours[f], ref[f])
    assert ours["nslices"] == ref["nslices"]
