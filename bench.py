#!/usr/bin/env python
"""PatchTable query throughput on B200.

Workload (default): the 1920x1080 synthetic match -- image a = 4 octaves of value noise + 20
rectangles, b = a warped by a smooth random flow (max 16 px) + N(0, 0.02) noise (seed 2) -- with
the reference's default parameters plus -speed 3 -coherence_spatial 4.  One step = one full query
(descriptor of a, table lookup, k-coherence unless the schedule caps it at none, propagation
passes, float64 NNF) against a table of b built once before warm-up.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --profile-case query|query-default|infer|build|build-c2  (short fixed runs for ncu)

Prints one JSON line (rank 0).  `value` is query patches per second of device time (one CUDA event
pair around each pt_table_lookup_device call) with a already
in device memory (L2 flushed between steps) at the fastest query schedule whose mean NNF distance
is within 1% of the reference's on this workload; `e2e` is the same metric through the public host
API (pt_table_lookup) with pinned host buffers, copies included.  config.learned compares the
learned-proposal query with the plain one at matched quality.  --impl reference times the
reference's own implementation (oracle/_ref, compiled from its sources) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="synthetic 1920x1080 match, -speed 3 -coherence_spatial 4", h=1080, w=1920, seed=2,
                switches="-speed 3 -coherence_spatial 4")
METRIC = "query patches/s at matched mean NNF dist (learned vs plain, 1 B200); build s"
UNIT = "patches/s"
L2_FLUSH_BYTES = 256 << 20
# query schedules (passes, first jump, pull candidates per patch; 0 = all); every one is timed and
# the fastest whose mean NNF distance is within 1% of the reference's is the measured one
# a fourth entry caps the k-coherence neighbours tried per patch (gpu_kc_max; -1 = none, the table
# step and the pulls alone); the table is the same in every case
SCHEDULES = [(1, 2, 1, -1), (1, 1, 1, -1), (1, 2, 2, -1), (2, 2, 1, -1), (1, 2, 1, 1), (1, 2, 1), (1, 1, 1), (1, 2, 2),
             (1, 2, 3), (1, 2, 0), (2, 2, 1), (2, 2, 2), (2, 2, 0), (3, 4, 0), (4, 8, 0)]
# learned-proposal comparison: schedules tried for both forms against the plain default's quality
LEARNED_SCHEDULES = [(1, 2, 0), (2, 2, 0), (2, 2, 2), (3, 4, 0), (4, 8, 0)]
PROPOSAL_WEIGHTS = os.path.join(ROOT, "patchtable_b200", "data", "proposal_weights.npy")


def reference_mean_dist():
    """Mean NNF distance of the reference (oracle/_ref, 1 thread) on this workload, recorded by
    tests/golden/make_golden.py."""
    with open(os.path.join(ROOT, "tests", "golden", "oracle_golden.json")) as f:
        g = json.load(f)["c2"]
    assert (g["h"], g["w"], g["seed"], g["switches"]) == (WORKLOAD["h"], WORKLOAD["w"], WORKLOAD["seed"], WORKLOAD["switches"])
    return g["mean_dist"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--profile-case", choices=["query", "query-default", "infer", "build", "build-c2"], default=None)
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """SM clock and clock-event reasons sampled through NVML (read-only) every millisecond while
    the timed region runs."""
    NAMES = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
             0x80: "hw_power_brake_slowdown"}

    def __init__(self, dev_index: int):
        self.samples = []
        self.stop_ev = threading.Event()
        self.th = None
        self.nv = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            try:
                uuid = str(torch.cuda.get_device_properties(dev_index).uuid)
                self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(dev_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.nv = pynvml
        except Exception:
            self.nv = None

    def _loop(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                self.samples.append((time.perf_counter(), nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
            except Exception:
                pass
            time.sleep(0.001)

    def start(self):
        if self.nv is not None:
            self.th = threading.Thread(target=self._loop, daemon=True)
            self.th.start()

    def stop(self, window=None):
        """Clock record of the samples inside `window` (perf_counter start, end) -- the timed
        region; when an NVML call is slow and fewer than 3 land there, the samples of the whole
        sampled stretch (warm-up lookups and timed region, the same load) are used and said so."""
        if self.nv is None or self.th is None:
            return None
        self.stop_ev.set()
        self.th.join(timeout=5)
        if not self.samples:
            return None
        inside = [x for x in self.samples if window is None or window[0] <= x[0] <= window[1]]
        used, span = ((inside, "timed region") if len(inside) >= 3 else
                      (self.samples, "timed region and the 0.25 s of warm-up lookups just before it"))
        reasons = sorted({n for _, _, r in used for bit, n in self.NAMES.items() if r & bit})
        return {"sm_mhz": statistics.median(m for _, m, _ in used), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(inside), "samples_used": len(used), "window": span,
                "source": "nvml, every 1 ms"}


def make_inputs():
    from patchtable_b200 import synth
    return synth.pair(WORKLOAD["h"], WORKLOAD["w"], WORKLOAD["seed"])


def cpu_baseline(a, b):
    """The reference's own lookup (oracle/_ref) on a bounded crop of the workload, host cores."""
    from oracle.oracle import REF_SO, Reference
    if not os.path.exists(REF_SO):
        return None
    cores = os.cpu_count() or 1
    h, w = 540, 960
    ac, bc = np.ascontiguousarray(a[:h, :w]), np.ascontiguousarray(b[:h, :w])
    ref = Reference()
    ref.srand(1)
    t = ref.build(WORKLOAD["switches"] + " -threads %d" % cores, bc)
    secs = []
    for _ in range(3):
        _, s = t.lookup(ac)
        secs.append(s)
    P = (h - 7) * (w - 7)
    return {"value": P / min(secs[1:]), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": "reference lookup (oracle/_ref, -threads %d) on the top-left %dx%d crop of the workload pair, "
                      "best of 2 timed lookups after 1 warm-up; table build %.1f s" % (cores, w, h, t.build_seconds)}


def run_reference(args, rank):
    """--impl reference: the reference implementation on the host cores, full workload."""
    if rank != 0:
        return
    from oracle.oracle import REF_SO, Reference, mean_dist
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libptref.so was not built (needs the reference sources)"}))
        return
    a, b = make_inputs()
    cores = os.cpu_count() or 1
    ref = Reference()
    ref.srand(1)
    t = ref.build(WORKLOAD["switches"] + " -threads %d" % cores, b)
    P = (a.shape[0] - 7) * (a.shape[1] - 7)
    for _ in range(args.warmup):
        t.lookup(a)
    secs = []
    md = None
    for _ in range(args.steps):
        ann, s = t.lookup(a)
        secs.append(s)
        md = mean_dist(ann)
    tot = sum(secs)
    val = P * args.steps / tot
    out = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1000 * tot / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": {"workload": WORKLOAD["name"], "patches_per_step": P, "threads": cores, "build_s": t.build_seconds,
                      "mean_nnf_dist": md},
           "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference",
                            "sample": "full workload, one reference lookup per step (PatchTable::lookup timer)"},
           "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def profile_case(name):
    """Short fixed runs of one kernel family, for ncu captures."""
    import torch
    import patchtable_b200 as ptb
    from patchtable_b200 import synth
    ctypes.CDLL(None).srand(1)
    st = torch.cuda.current_stream().cuda_stream
    if name in ("build", "build-c2"):
        h, w = (540, 960) if name == "build" else (WORKLOAD["h"], WORKLOAD["w"])
        a, b = synth.pair(h, w, 2)
        t = ptb.PatchTable(ptb.PatchTableParams(WORKLOAD["switches"]), b)
        torch.cuda.synchronize()
        print("profile case %s: %d cells, stages %s" % (name, t.shape()[1], t.build_profile()))
        return
    if name in ("query", "query-default"):
        a, b = make_inputs()
        H, W = a.shape[:2]
        p = ptb.PatchTableParams(WORKLOAD["switches"])
        t = ptb.PatchTable(p, b)
        if name == "query":
            p.set_schedule(SCHEDULES[0])
            p.gpu_tile = 128         # the timed run's sweep picks 128 or 64 on B200 (within 1 %)
        da = torch.from_numpy(a).cuda()
        dann = torch.empty((H - 7) * (W - 7) * 3, dtype=torch.float64, device="cuda")
        for _ in range(2):
            t.lookup_device(da.data_ptr(), H, W, dann.data_ptr(), st)
        torch.cuda.synchronize()
        print("profile case %s: mean NNF dist %.5f" % (name, float(dann.view(-1, 3)[:, 2].clamp(min=0).sqrt().mean())))
    else:
        from patchtable_b200.proposal import ProposalNet
        h, w = 540, 960
        a, b = synth.pair(h, w, 6000)
        t = ptb.PatchTable(ptb.PatchTableParams(WORKLOAD["switches"]), b)
        net = ProposalNet(seed=0)
        P = (h - 7) * (w - 7)
        da = torch.from_numpy(a).cuda()
        cand = torch.empty((P, 8), dtype=torch.int32, device="cuda")
        conf = torch.empty(P, dtype=torch.float32, device="cuda")
        for _ in range(3):
            t.proposal_infer(net, da.data_ptr(), h, w, cand.data_ptr(), conf.data_ptr(), 0, st)
        torch.cuda.synchronize()
        print("profile case infer: mean confidence %.5f" % float(conf.mean()))


def timed_schedule(table, sched, da, H, W, dann, sptr, flush, reps=3, net=None):
    """(best device ms of `reps` lookups after one untimed, mean NNF dist) of one schedule: one CUDA
    event pair around each production call (pt_table_lookup_device or its learned form)."""
    import torch
    from patchtable_b200.metrics import get_mean_dist
    p = table.params
    p.set_schedule(sched)
    stream = torch.cuda.current_stream()
    best = None
    for i in range(reps + 1):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if net is None:
            table.lookup_device(da.data_ptr(), H, W, dann.data_ptr(), sptr)
        else:
            table.lookup_learned_device(net, da.data_ptr(), H, W, dann.data_ptr(), sptr)
        e1.record(stream)
        e1.synchronize()
        if i > 0:
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
    torch.cuda.synchronize()
    return best, get_mean_dist(dann.cpu().numpy())


def learned_comparison(table, da, H, W, dann, sptr, flush, P):
    """The learned-proposal query against the plain one at the plain default schedule's quality."""
    if not os.path.exists(PROPOSAL_WEIGHTS):
        return {"unavailable": "no trained proposal weights at patchtable_b200/data/proposal_weights.npy"}
    import patchtable_b200 as ptb
    from patchtable_b200.proposal import ProposalNet
    net = ProposalNet.load(PROPOSAL_WEIGHTS)
    _, target = timed_schedule(table, (0, 0, 0), da, H, W, dann, sptr, flush, reps=1)
    bar = 1.01 * target
    out = {"quality_bar": {"mean_nnf_dist": bar, "rule": "within 1% of the plain default schedule's mean"}}
    rows = {}
    for label, thr in (("plain", None), ("learned_threshold_0.5", 0.5), ("learned_threshold_0", 0.0)):
        best = None
        tried = {}
        for sched in LEARNED_SCHEDULES:
            if thr is None:
                ms, md = timed_schedule(table, sched, da, H, W, dann, sptr, flush)
            else:
                net.configure(thr, False)
                ms, md = timed_schedule(table, sched, da, H, W, dann, sptr, flush, net=net)
            tried[ptb.schedule_name(sched)] = {"ms": ms, "mean_nnf_dist": md}
            if md <= bar and (best is None or ms < best[0]):
                best = (ms, sched, md)
        rows[label] = {"patches_per_s": P / (best[0] / 1000.0) if best else None,
                       "schedule": ptb.schedule_name(best[1]) if best else None,
                       "mean_nnf_dist": best[2] if best else None, "tried": tried}
    out.update(rows)
    if rows["plain"]["patches_per_s"]:
        for k in ("learned_threshold_0.5", "learned_threshold_0"):
            if rows[k]["patches_per_s"]:
                rows[k]["vs_plain"] = rows[k]["patches_per_s"] / rows["plain"]["patches_per_s"]
    net.close()
    return out


def _event_ms(fn, reps):
    """Best device time (CUDA events on the current stream) of `reps` calls of fn after one warm-up."""
    import torch
    st = torch.cuda.current_stream()
    fn()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best


def uneven_batch_measure():
    """64 query images with sides uniform in [128, 2048] against one 1920x1080 table: the batched
    query (autotuned patches per CTA, replayed as one captured CUDA graph) against one
    pt_table_lookup_device call per image, at 2, 4 and 8 propagation passes."""
    import torch
    import patchtable_b200 as ptb
    from patchtable_b200 import synth
    from patchtable_b200.metrics import get_mean_dist
    table_img, queries = synth.uneven_batch()
    params = ptb.PatchTableParams(WORKLOAD["switches"])
    ctypes.CDLL(None).srand(1)
    table = ptb.PatchTable(params, table_img)
    qb = table.batch([q.shape[:2] for q in queries])
    rgb = torch.empty(qb.pixels * 3, dtype=torch.float32, device="cuda")
    for q, o in zip(queries, qb.pixel_offset):
        rgb[3 * o:3 * o + q.size] = torch.from_numpy(q.ravel()).cuda()
    ann = torch.empty(qb.patches * 3, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    P = qb.patches

    def per_image():
        for q, po, qo in zip(queries, qb.pixel_offset, qb.patch_offset):
            table.lookup_device(rgb.data_ptr() + 12 * int(po), q.shape[0], q.shape[1], ann.data_ptr() + 24 * int(qo), st)

    rows = {}
    for sched in ((2, 2, 0), (4, 8, 0), (8, 8, 0), SCHEDULES[0]):
        params.set_schedule(sched)
        best, tune = qb.autotune(rgb.data_ptr(), ann.data_ptr(), st)
        qb.capture(rgb.data_ptr(), ann.data_ptr(), st)
        g_ms = _event_ms(lambda: qb.replay(st), 3)
        md = get_mean_dist(ann.view(-1, 3).cpu().numpy()[None])
        pi_ms = _event_ms(per_image, 2)
        rows[ptb.schedule_name(sched)] = {
            "graph_patches_per_s": P / (g_ms / 1000.0), "per_image_patches_per_s": P / (pi_ms / 1000.0),
            "speedup": pi_ms / g_ms, "mean_nnf_dist": md, "patches_per_cta": best,
            "autotune_ms": {str(k): v for k, v in tune.items()}}
    qb.close()
    return {"images": len(queries), "patches": P, "table_image": [1080, 1920],
            "workload": "64 queries, sides U[128, 2048], crops of the warped 2048^2 base (seeds 4000+i)",
            "schedules": rows}


def uneven_batch_sharded(dev, world, rank):
    """The 64-image batch split by image over the ranks (cost-balanced by patch count): every rank
    builds the table and answers its share as one batched query (graph replay, 1 pass / jump 2 /
    1 pull candidate); the whole job's rate is all patches over the slowest rank's time."""
    import torch
    import patchtable_b200 as ptb
    from patchtable_b200 import replicas, synth
    table_img, queries = synth.uneven_batch()
    costs = [(q.shape[0] - 7) * (q.shape[1] - 7) for q in queries]
    mine = replicas.shard_by_cost(costs, world)[rank]
    params = ptb.PatchTableParams(WORKLOAD["switches"])
    ctypes.CDLL(None).srand(1)
    table = ptb.PatchTable(params, table_img)
    params.set_schedule(SCHEDULES[0])
    qs = [queries[i] for i in mine]
    qb = table.batch([q.shape[:2] for q in qs])
    rgb = torch.empty(qb.pixels * 3, dtype=torch.float32, device=dev)
    for q, o in zip(qs, qb.pixel_offset):
        rgb[3 * o:3 * o + q.size] = torch.from_numpy(q.ravel()).to(dev)
    ann = torch.empty(qb.patches * 3, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    qb.set_tile(32)
    qb.capture(rgb.data_ptr(), ann.data_ptr(), st)
    replicas.barrier()
    ms = _event_ms(lambda: qb.replay(st), 3)
    slow = replicas.max_over_ranks(ms, dev)
    qb.close()
    table.close()
    return {"images": len(queries), "patches": sum(costs), "ranks": world, "my_images": len(mine),
            "slowest_rank_ms": slow, "patches_per_s": sum(costs) / (slow / 1000.0),
            "split": "by image, most patches first to the least-loaded rank"}


def one_vs_many_measure():
    """One 1024x768 query against 10 database images (sides U[256, 2048]) packed into one atlas
    table, seam-straddling patches excluded by the allowed mask."""
    import torch
    import patchtable_b200 as ptb
    from patchtable_b200 import synth
    from patchtable_b200.metrics import get_mean_dist
    query, atlas, allowed, boxes = synth.one_vs_many()
    params = ptb.PatchTableParams(WORKLOAD["switches"])
    ctypes.CDLL(None).srand(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    table = ptb.PatchTable(params, atlas, allowed_patches=allowed)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    build_stage_ms = table.build_profile()
    H, W = query.shape[:2]
    P = (H - 7) * (W - 7)
    da = torch.from_numpy(query).cuda()
    dann = torch.empty((H - 7, W - 7, 3), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rows = {}
    for sched in (SCHEDULES[0], (0, 0, 0)):
        params.set_schedule(sched)
        ms = _event_ms(lambda: table.lookup_device(da.data_ptr(), H, W, dann.data_ptr(), st), 3)
        ann = dann.cpu().numpy()
        ok = bool(np.all(allowed[ann[..., 1].astype(int), ann[..., 0].astype(int)] == 1))
        rows[ptb.schedule_name(sched)] = {"patches_per_s": P / (ms / 1000.0), "ms": ms, "mean_nnf_dist": get_mean_dist(ann),
                                    "all_matches_allowed": ok}
    table.close()
    return {"query": [H, W], "atlas": list(atlas.shape[:2]), "database_images": len(boxes),
            "allowed_patches": int(allowed.sum()), "build_s": build_s, "build_stage_ms": build_stage_ms, "schedules": rows}


def main():
    args = parse()
    from patchtable_b200 import replicas
    rank, world, local = replicas.env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import patchtable_b200 as ptb
    from patchtable_b200.metrics import get_mean_dist as mean_dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.profile_case:
        profile_case(args.profile_case)
        return
    replicas.init("nccl", dev)

    a, b = make_inputs()
    H, W = a.shape[:2]
    P = (H - 7) * (W - 7)
    params = ptb.PatchTableParams(WORKLOAD["switches"])
    # the first table of a process also loads the library's kernels onto the device: time it, then
    # time the build again as every later table of the process runs it
    ctypes.CDLL(None).srand(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    first = ptb.PatchTable(params, b)
    torch.cuda.synchronize()
    first_build_s = time.perf_counter() - t0
    first.close()
    del first
    # warm builds: the median of three (the host's page-locking, allocation and thread start-up
    # make single builds vary); the last table answers the queries
    builds = []
    table = None
    for _ in range(3):
        if table is not None:
            table.close()
        ctypes.CDLL(None).srand(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        table = ptb.PatchTable(params, b)
        torch.cuda.synchronize()
        builds.append((time.perf_counter() - t0, table.build_profile()))
    build_s, build_stage_ms = sorted(builds, key=lambda x: x[0])[1]
    build_s_all = [x[0] for x in builds]

    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    da = torch.from_numpy(a).to(dev)
    dann = torch.empty((H - 7, W - 7, 3), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    # the fastest schedule within 1% of the reference's mean NNF distance
    ref_md = reference_mean_dist()
    sched_md = {}
    chosen = None
    for sched in SCHEDULES:
        ms, m = timed_schedule(table, sched, da, H, W, dann, sptr, flush)
        sched_md[ptb.schedule_name(sched)] = {"ms": ms, "mean_nnf_dist": m}
        if m <= 1.01 * ref_md and (chosen is None or ms < chosen[0]):
            chosen = (ms, sched)
    chosen = chosen[1] if chosen else SCHEDULES[-1]
    chosen = SCHEDULES[int(replicas.agree(SCHEDULES.index(chosen), dev))]   # every rank runs rank 0's choice
    # query patches per CTA: the results do not depend on it, only the time does
    tile_ms = {}
    for tile in (32, 64, 128, 256):
        params.gpu_tile = tile
        tile_ms[tile], _ = timed_schedule(table, chosen, da, H, W, dann, sptr, flush)
    params.gpu_tile = int(replicas.agree(min(tile_ms, key=tile_ms.get), dev))
    params.set_schedule(chosen)
    # warm-up: at least W lookups and at least 0.25 s of them, with the clocks sampled from here on
    # (an NVML query can take longer than a millisecond, and the timed region is short)
    clocks = Clocks(local)
    clocks.start()
    tw_start = time.perf_counter()
    n_warm = 0
    while n_warm < max(args.warmup, 3) or time.perf_counter() - tw_start < 0.25:
        flush.zero_()
        table.lookup_device(da.data_ptr(), H, W, dann.data_ptr(), sptr)
        n_warm += 1
        if n_warm % 16 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()

    # the timed region: one CUDA event pair around each production call (pt_table_lookup_device)
    replicas.barrier()
    torch.cuda.synchronize()
    ptb.reset_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    tw0 = time.perf_counter()
    for i in range(args.steps):
        flush.zero_()                       # evict L2 between steps (outside the timed events)
        ev[i][0].record(stream)
        table.lookup_device(da.data_ptr(), H, W, dann.data_ptr(), sptr)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - tw0
    launches = ptb.launch_count()
    clk = clocks.stop((tw0, tw0 + wall))
    replicas.barrier()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    tot_ms = replicas.max_over_ranks(sum(step_ms), dev)
    value = replicas.whole_job_rate(P * args.steps, tot_ms / 1000.0, world)
    md_timed = mean_dist(dann.cpu().numpy())
    md = md_timed                           # every step returns the same field

    # per-kernel breakdown for the roofline: the same steps again through the diagnostic entry
    # point, which records a CUDA event after every kernel on the launching stream
    stages, ctrs = {k: 0.0 for k in ptb.PatchTable.STAGES}, {}
    for i in range(args.steps):
        flush.zero_()
        st, c = table.lookup_profile(da.data_ptr(), H, W, dann.data_ptr(), sptr)
        for k, v in st.items():
            stages[k] += v
        for k, v in c.items():
            ctrs[k] = ctrs.get(k, 0) + v
    torch.cuda.synchronize()

    # end-to-end through the public host API with pinned buffers
    a_pin = torch.from_numpy(a).pin_memory()
    ann_pin = torch.empty((H - 7, W - 7, 3), dtype=torch.float64).pin_memory()
    a_np, ann_np = a_pin.numpy(), ann_pin.numpy()
    for _ in range(max(args.warmup, 3)):
        table.lookup(a_np, out=ann_np)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        table.lookup(a_np, out=ann_np)
        e2e_s.append(time.perf_counter() - t1)
    e2e = replicas.whole_job_rate(P, replicas.max_over_ranks(sum(e2e_s) / len(e2e_s), dev), world)
    md_e2e = mean_dist(ann_np)
    h2d_bytes, d2h_bytes = table.last_transfer()
    # the transfer floor of e2e: the same bytes copied alone between pinned host and device memory
    h2d_ms = _event_ms(lambda: da.copy_(a_pin, non_blocking=True), 5)
    dsrc = torch.empty(d2h_bytes // 4, dtype=torch.float32, device=dev)
    hdst = torch.empty(d2h_bytes // 4, dtype=torch.float32).pin_memory()
    d2h_ms = _event_ms(lambda: hdst.copy_(dsrc, non_blocking=True), 5)
    del dsrc, hdst
    e2e_mean_ms = 1000 * sum(e2e_s) / len(e2e_s)
    transfer = {"h2d_bytes": h2d_bytes, "d2h_bytes": d2h_bytes, "h2d_ms": h2d_ms, "d2h_ms": d2h_ms,
                "h2d_gbs": h2d_bytes / h2d_ms / 1e6, "d2h_gbs": d2h_bytes / d2h_ms / 1e6,
                "floor_ms": max(h2d_ms, d2h_ms), "floor_frac_of_e2e": max(h2d_ms, d2h_ms) / e2e_mean_ms,
                "note": "floor = the slower of the two copies alone (perfect overlap of upload, kernels and "
                        "download); the lookup downloads 8 B per patch and widens to float64 on the host"}

    # the library's default schedule on the same workload, for reference
    dflt_ms, dflt_md = timed_schedule(table, (0, 0, 0), da, H, W, dann, sptr, flush, reps=max(3, args.steps // 2))
    default_sched = {"patches_per_s": P / (dflt_ms / 1000.0), "mean_nnf_dist": dflt_md}
    learned = None
    if not args.no_learned and rank == 0:
        learned = learned_comparison(table, da, H, W, dann, sptr, flush, P)
    params.set_schedule(chosen)

    # roofline of the dominant query kernel.  Both query kernels are limited by the L1TEX data
    # pipe (wavefronts of the scattered 8x8 patch gathers) long before HBM; the HBM figure counts
    # the kernel's algorithmic bytes, the fp32 figure its SSD arithmetic.
    hbm, peak_kind = peaks()
    passes = chosen[0]
    dom = max(("choose", "pull"), key=lambda k: stages[k])
    per_launch_ms = stages[dom] / (args.steps * passes)
    # bytes per patch averaged over the passes: the first pass reads no state (8 B), the last pull
    # writes the float64 NNF (24 B) in place of the next state (8 B)
    later = (passes - 1) / passes
    # choose: a 16, table entry 4, b pixels 16, chosen 12, and 8 per k-coherence entry it reads
    kc_cap = chosen[3] if len(chosen) > 3 else 0
    kc_n = params.kcoherence if kc_cap == 0 else (0 if kc_cap < 0 else min(kc_cap, params.kcoherence))
    alg_bytes = {"choose": 48 + 8 * kc_n + 8 * later, "pull": 40 + 8 * later + (24 + 8 * (passes - 1)) / passes}[dom] * P
    achieved = alg_bytes / (per_launch_ms / 1000.0) / 1e9
    # DRAM traffic and the L1 data-pipe share cannot be measured inside this run: they come from
    # the committed ncu summary of the same kernel and schedule, which names its source revision
    traffic, l1, prof_src = None, None, {"file": "profiles/query_%s_c2.md" % dom, "source_revision": None}
    try:
        with open(os.path.join(ROOT, "profiles", "query_%s_c2.md" % dom)) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    traffic = float(line.split(":")[1])
                if line.startswith("l1tex_wavefront_pct_of_peak:"):
                    l1 = float(line.split(":")[1])
                if line.startswith("source_revision:"):
                    prof_src["source_revision"] = line.split(":", 1)[1].strip()
    except OSError:
        pass
    rows = ctrs.get(dom + "_rows", 0)
    fp32_tflops = rows * 72 / (stages[dom] / 1000.0) / 1e12

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(a, b)
    c4 = c3 = c4s = None
    if not args.no_batch:
        del flush
        torch.cuda.empty_cache()
        if world > 1:
            c4s = uneven_batch_sharded(dev, world, rank)
        elif rank == 0:
            c4 = uneven_batch_measure()
            c3 = one_vs_many_measure()

    replicas.finish()
    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generator, patchtable_b200/synth.py)",
        "config": {"workload": WORKLOAD["name"], "patches_per_step": P, "image": [H, W], "table_image": list(b.shape[:2]),
                   "build_s": build_s, "build_s_all": build_s_all, "build_stage_ms": build_stage_ms,
                   "first_build_s": first_build_s, "mean_nnf_dist": md, "mean_nnf_dist_e2e": md_e2e,
                   "e2e_ms": {"mean": 1000 * sum(e2e_s) / len(e2e_s), "median": 1000 * float(np.median(e2e_s)),
                              "min": 1000 * min(e2e_s), "max": 1000 * max(e2e_s), "calls": len(e2e_s)},
                   "reference_mean_nnf_dist": ref_md,
                   "schedule": {"passes": chosen[0], "first_jump": chosen[1], "pull_max": chosen[2],
                                "kc_max": chosen[3] if len(chosen) > 3 else 0, "tried": sched_md,
                                "patches_per_cta": params.gpu_tile, "patches_per_cta_ms": {str(k): v for k, v in tile_ms.items()},
                                "rule": "fastest schedule with mean NNF dist <= 1.01 x the reference's on this workload"},
                   "library_default_schedule": default_sched, "learned": learned,
                   "uneven_batch": c4, "uneven_batch_sharded": c4s, "one_vs_many": c3, "mean_nnf_dist_timed": md_timed,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": "replicas" if world > 1 else "single",
                   "timing": "one CUDA event pair around each pt_table_lookup_device call on its stream",
                   "step_ms": {"min": min(step_ms), "median": float(np.median(step_ms)), "max": max(step_ms)},
                   "stage_ms_per_step": {k: v / args.steps for k, v in stages.items()},
                   "stage_ms_source": "pt_table_lookup_profile (an event after every kernel), same steps, run after the timed region",
                   "e2e_transfer": transfer, "wall_ms_per_step": 1000 * wall / args.steps,
                   "ssd_candidates_per_patch": {k: ctrs.get(k + "_cand", 0) / (args.steps * P) for k in ("choose", "pull")}},
        "roofline": {"bound": "hbm", "kernel": "k_" + dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "traffic_source": prof_src, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "limiter": {"unit": "L1TEX data-pipe wavefronts", "pct_of_peak_ncu": l1},
                     "fp32": {"achieved_tflops": fp32_tflops, "flop_per_ssd_row": 72,
                              "ssd_rows_per_launch": rows / (args.steps * passes)}},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d_bytes), "d2h_bytes_per_step": int(d2h_bytes)},
        "gpu_launches": int(launches),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
