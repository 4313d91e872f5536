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


def test_gpu_schedule_switches():
    """The GPU schedule switches (no reference counterpart) parse, default to 0 and leave every
    reference field as the reference sets it; set_schedule / schedule_name round-trip."""
    base = ptb.PatchTableParams("-speed 3 -coherence_spatial 4")
    p = ptb.PatchTableParams("-speed 3 -coherence_spatial 4 -gpu_prop_passes 2 -gpu_jump 4 -gpu_pull_max 3 "
                             "-gpu_kc_max -1 -gpu_tile 64 -gpu_bands 12")
    assert (p.gpu_prop_passes, p.gpu_jump, p.gpu_pull_max, p.gpu_kc_max, p.gpu_tile, p.gpu_bands) == (2, 4, 3, -1, 64, 12)
    for f in PARAM_FIELDS:
        assert getattr(p, f) == getattr(base, f), f
    assert (base.gpu_prop_passes, base.gpu_jump, base.gpu_pull_max, base.gpu_kc_max) == (0, 0, 0, 0)
    base.set_schedule((1, 2, 1, -1))
    assert (base.gpu_prop_passes, base.gpu_jump, base.gpu_pull_max, base.gpu_kc_max) == (1, 2, 1, -1)
    base.set_schedule((4, 8, 0))
    assert base.gpu_kc_max == 0
    assert ptb.schedule_name((1, 2, 1, -1)) == "1/2/1/-1" and ptb.schedule_name((1, 2, 1)) == "1/2/1"
    assert ptb.schedule_name((3, 4, 0, 0)) == "3/4/0"
