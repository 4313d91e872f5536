"""Generates tests/golden/oracle_golden.json from the reference's own implementation.

Runs the reference sources compiled in place (oracle/_ref/libptref.so) on seeded synthetic pairs
and records digests of every intermediate the parity tests compare (descriptor, partition, table
after the DT, k-coherence set, NNF) plus mean NNF distances.  The CPU tests recompute the same
quantities with the restatement (oracle/pt_oracle.cpp) and require identical digests, which pins
the restatement to the reference on machines where the reference cannot be built.

Also records the reference's result on the repository's sample pair patchtable/vidpair0 (the pair
of patchtable/match_ours_full.txt:4, mean_dist 0.130757 at -speed 3 with the original FLANN).

Needs the reference checkout ($PATCHTABLE_REFERENCE, else the location oracle/Makefile reads) and a
built oracle/_ref:
    python tests/golden/make_golden.py          every entry
    python tests/golden/make_golden.py --c2     only the 1920x1080 entry (digests of every stage)
    python tests/golden/make_golden.py --add    append the entries of CASES that the file lacks
"""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference, mean_dist  # noqa: E402
from patchtable_b200 import synth  # noqa: E402

CASES = [
    dict(name="tiny_64x48", h=48, w=64, seed=11, switches="-limit 1"),
    dict(name="small_96x80_coh4", h=80, w=96, seed=12, switches="-limit 1 -coherence_spatial 4"),
    dict(name="small_120x90_k4", h=90, w=120, seed=13, switches="-limit 1 -kcoherence 4 -prop_iters 3"),
    dict(name="small_100x70_speed6", h=70, w=100, seed=15, switches="-speed 6 -limit 0.5"),
    dict(name="c1_320x240", h=240, w=320, seed=1, switches=""),
    dict(name="c1_320x240_coh4", h=240, w=320, seed=1, switches="-coherence_spatial 4"),
    dict(name="dt_downsample_100x80", h=80, w=100, seed=16, switches="-limit 1 -dt_algo downsample"),
    dict(name="dt_hybrid_110x90_nd8", h=90, w=110, seed=17, switches="-limit 0.3 -ndims 8 -dt_algo hybrid"),
    dict(name="dt_euclidean_90x120_nd3", h=120, w=90, seed=18,
         switches="-limit 2 -ndims 3 -coherence_spatial 4 -dt_algo euclidean"),
    dict(name="ntables3_90x60", h=60, w=90, seed=19, switches="-limit 1 -ntables 3 -coherence_spatial 2"),
    dict(name="ntables2_ratio4_k3_70x80", h=80, w=70, seed=20, switches="-limit 0.5 -ntables 2 -table_ratio 4 -kcoherence 3"),
    dict(name="lab_100x80_k2", h=80, w=100, seed=24, switches="-limit 1 -colorspace lab -kcoherence 2"),
    dict(name="dt_brute_80x60", h=60, w=80, seed=25, switches="-limit 0.003 -dt_algo brute -coherence_spatial 2"),
    dict(name="dt_brute_g2_70x50", h=50, w=70, seed=26, switches="-limit 0.0008 -grid_ndims 2 -dt_algo brute"),
    # The same pair and switches as tiny_64x48: both options leave the reference's table unchanged.
    dict(name="noop_switches_64x48", h=48, w=64, seed=11, switches="-limit 1 -randomize_dt 1 -populate_nearest 0"),
    # -dim_algo pca: the reference's own patch sampling and projection (patch_pca.h) around the
    # cv::PCA stand-in of oracle/pca_jacobi.h.
    dict(name="pca_160x120", h=120, w=160, seed=11, switches="-dim_algo pca -limit 1"),
    dict(name="pca_nd8_k2_130x100", h=100, w=130, seed=12, switches="-dim_algo pca -ndims 8 -kcoherence 2 -limit 2"),
    dict(name="pca_nd4_nomean_70x90", h=90, w=70, seed=13,
         switches="-dim_algo pca -ndims 4 -pca_subtract_mean 0 -pca_samples 300 -limit 0.5"),
    dict(name="pca_nd12_rgb_110x80", h=80, w=110, seed=14, switches="-dim_algo pca -ndims 12 -colorspace rgb -limit 3"),
    dict(name="pca_lab_120x90", h=90, w=120, seed=15, switches="-dim_algo pca -colorspace lab -limit 1"),
    # sampled k-coherence: train set every 2nd patch, queries every 2nd / 3rd pixel, knn reset segments
    dict(name="kc_steps_90x70", h=70, w=90, seed=27,
         switches="-limit 0.5 -kcoherence 3 -kcoherence_step 2 -flann_build_step 2 -flann_reset_step 3"),
    dict(name="kc_reset1_90x70", h=70, w=90, seed=27, switches="-limit 0.5 -kcoherence 2 -flann_reset_step 1"),
]
C2 = dict(name="c2_1920x1080_coh4", h=1080, w=1920, seed=2, switches="-speed 3 -coherence_spatial 4")
# Descriptor mode (is_descriptor): synth.descriptor_pair inputs.  Three channels are left out: the
# reference's fourth SSE lane then reads padding that Array::resize leaves uninitialised
# (solver/array.h:286-287).
DESC_CASES = [
    dict(name="desc8_60x80", h=60, w=80, c=8, seed=41, switches="-limit 0.2 -is_descriptor 1"),
    dict(name="desc6_k4_50x70", h=50, w=70, c=6, seed=42, switches="-limit 0.2 -kcoherence 4 -is_descriptor 1"),
    dict(name="desc12_g6_45x66", h=45, w=66, c=12, seed=43, switches="-limit 0.3 -grid_ndims 6 -is_descriptor 1"),
    dict(name="desc7_padded_52x61", h=52, w=61, c=7, seed=44,
         switches="-limit 0.1 -is_descriptor 1 -descriptor_padded 1 -coherence_spatial 2"),
    dict(name="desc15_40x48", h=40, w=48, c=15, seed=45, switches="-limit 0.5 -is_descriptor 1"),
]


def digest(arr) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()


def wh0_digest(wh0, case: dict) -> str:
    """Digest of a descriptor image.  apply_patch_pca writes only the patch positions
    (patch_pca.h:82-83) and leaves the 7-pixel border of its freshly resized array uninitialised
    (solver/array.h:286-287), so PCA descriptors are compared on the patch positions only."""
    if "-dim_algo pca" in case["switches"]:
        return digest(wh0[7:case["h"], 7:case["w"]])
    return digest(wh0)


def run_case(ref: Reference, case: dict, full: bool = True) -> dict:
    a, b = synth.pair(case["h"], case["w"], case["seed"])
    ref.srand(1)
    t = ref.build(case["switches"], b)
    ann, _ = t.lookup(a)
    out = dict(case)
    out["mean_dist"] = mean_dist(ann)
    out["ann"] = digest(ann)
    if full:
        ns, _ = t.shape()
        out["nslices"] = ns
        out["add_count"] = t.add_count()
        out["wh0"] = wh0_digest(t.wh0(), case)
        out["table"] = digest(t.table())
        parts = [t.partition(d) for d in range(len(ns))]
        out["partition"] = digest(np.concatenate([np.concatenate([p["centers"], p["lsizes"], p["rsizes"],
                                                                  p["to_bin"].view(np.float32), [p["min"], p["max"], p["range"]]])
                                                  for p in parts]))
        if t.params["kcoherence"] > 0:
            kp, kd = t.kcoherence()
            out["kcoh_pos"] = digest(kp)
            out["kcoh_dist"] = digest(kd)
    return out


def run_desc_case(ref: Reference, case: dict) -> dict:
    a, b = synth.descriptor_pair(case["h"], case["w"], case["c"], case["seed"])
    ref.srand(1)
    t = ref.build(case["switches"], b)
    ann, _ = t.lookup(a)
    out = dict(case)
    out["nslices"] = t.shape()[0]
    out["table"] = digest(t.table())
    if t.params["kcoherence"] > 0:
        kp, kd = t.kcoherence()
        out["kcoh_pos"] = digest(kp)
        out["kcoh_dist"] = digest(kd)
    out["ann"] = digest(ann)
    out["mean_dist"] = mean_dist(ann)
    return out


def reference_dir() -> str:
    env = os.environ.get("PATCHTABLE_REFERENCE")
    if env:
        return env
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"], stdout=subprocess.PIPE,
                       text=True, check=True)
    return r.stdout.strip()


def vidpair0(ref: Reference) -> dict:
    from PIL import Image
    base = os.path.join(reference_dir(), "patchtable", "vidpair0")

    def load(fn):
        # load_color_image for PNG: (real)(px * (1/255.0)), solver/array.h:1676-1680
        px = np.asarray(Image.open(os.path.join(base, fn)).convert("RGB"), dtype=np.float64)
        return (px * (1.0 / 255.0)).astype(np.float32)
    a, b = load("a.png"), load("b.png")
    ref.srand(1)
    t = ref.build("-speed 3", b)
    ann, _ = t.lookup(a)
    return dict(name="vidpair0_speed3", h=a.shape[0], w=a.shape[1], switches="-speed 3",
                mean_dist=mean_dist(ann), published_mean_dist=0.130757)


def main():
    ref = Reference()
    ref.set_threads(1)          # do_dt_brute shares one grid_index vector across its OpenMP loop (patchtable.h:2370-2376)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.json")
    if "--c2" in sys.argv:
        with open(path) as f:
            res = json.load(f)
        res["c2"] = run_case(ref, C2, full=True)
    elif "--add" in sys.argv:
        with open(path) as f:
            res = json.load(f)
        have = {c["name"] for c in res["cases"]}
        res["cases"] += [run_case(ref, c) for c in CASES if c["name"] not in have]
    else:
        res = {"cases": [run_case(ref, c) for c in CASES]}
        res["desc"] = [run_desc_case(ref, c) for c in DESC_CASES]
        res["c2"] = run_case(ref, C2, full=True)
        res["vidpair0"] = vidpair0(ref)
    with open(path, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({c["name"]: c["mean_dist"] for c in res["cases"] + [res["c2"], res["vidpair0"]]}, indent=1))


if __name__ == "__main__":
    main()
