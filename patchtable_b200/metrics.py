"""NNF quality metrics of the reference driver (patchtable/patchtable_main.cpp:90-101)."""
import numpy as np


def get_mean_dist(ann) -> float:
    """Mean over patches of sqrt(max(NNF_DIST, 0)), patchtable_main.cpp:90-101."""
    d = np.maximum(np.asarray(ann)[..., 2], 0.0)
    return float(np.sqrt(d).mean())
