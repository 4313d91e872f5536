"""Learned proposal network: training on the GPU, evaluation, and the learned query.

There is no counterpart in the reference.  The network (16 -> 128 -> ReLU -> 128 -> ReLU -> 32,
BF16 weights and activations, FP32 accumulation) maps a query patch's descriptor to a distribution
over table cells, factorised over the table's grid dimensions: for each dimension it scores the
bin offset -2..+2 of the match from the query patch's own bin.  The query scores the 8 most
probable cells' stored patches with the exact SSD; patches whose most probable cell has
probability below the threshold (0.5) keep the plain candidates (table cell + k-coherence).

Training data is the plain method's own output: for each seeded synthetic pair
(patchtable_b200.synth), a table of b with the query parameters, a plain lookup of a, and per query
patch the features and the bin offsets of the matched b patch (pt_table_proposal_samples).  Every
forward and backward product runs in the library's tcgen05 GEMM kernels; torch only holds device
memory and shuffles sample indices.

    python -m patchtable_b200.proposal train --pairs 200 --size 240x320 --out weights.npy
    python -m patchtable_b200.proposal eval --weights weights.npy --heldout 20 --size 1080x1920
    python -m patchtable_b200.proposal ablation --weights weights.npy --heldout 5 --out ablation.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time

import numpy as np

from . import PatchTable, PatchTableError, PatchTableParams, _check, lib, synth

DEFAULT_SWITCHES = "-speed 3 -coherence_spatial 4"
TRAIN_SEEDS = tuple(range(5000, 5200))
HELDOUT_SEEDS = tuple(range(6000, 6020))
IN, HIDDEN, OUT, DIMS, CLASSES, TOPK = 16, 128, 32, 6, 5, 8


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise PatchTableError(3, "the proposal network needs a CUDA device")
    return torch


def num_params() -> int:
    return int(lib().pt_proposal_num_params())


def param_slices():
    """Views of the parameter vector: W1 [128 x 16], b1, W2 [128 x 128], b2, W3 [32 x 128], b3."""
    shapes = [("W1", (HIDDEN, IN)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
              ("W3", (OUT, HIDDEN)), ("b3", (OUT,))]
    out, o = {}, 0
    for name, shp in shapes:
        n = int(np.prod(shp))
        out[name] = (o, shp)
        o += n
    assert o == num_params()
    return out


def unpack(vec: np.ndarray) -> dict:
    return {k: vec[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in param_slices().items()}


class ProposalNet:
    """pt_proposal: FP32 master parameters and AdamW state on the device."""

    def __init__(self, seed: int = 0, params: np.ndarray | None = None, threshold: float = 0.5,
                 kcoh_confident: bool = False):
        h = C.c_void_p()
        _check(lib().pt_proposal_create(C.c_uint32(seed), C.byref(h)))
        self._h = h
        if params is not None:
            self.set_params(params)
        self.configure(threshold, kcoh_confident)

    @property
    def handle(self):
        if not self._h or not self._h.value:
            raise PatchTableError(1, "proposal network is closed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().pt_proposal_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, threshold: float = 0.5, kcoh_confident: bool = False) -> None:
        self.threshold, self.kcoh_confident = float(threshold), bool(kcoh_confident)
        _check(lib().pt_proposal_configure(self.handle, C.c_float(threshold), int(kcoh_confident)))

    def params(self) -> np.ndarray:
        out = np.empty(num_params(), np.float32)
        _check(lib().pt_proposal_get_params(self.handle, out))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.shape != (num_params(),):
            raise PatchTableError(1, "expected %d parameters, got %s" % (num_params(), p.shape))
        _check(lib().pt_proposal_set_params(self.handle, p))

    def save(self, path: str) -> None:
        np.save(path, self.params())

    @classmethod
    def load(cls, path: str, **kw) -> "ProposalNet":
        return cls(params=np.load(path), **kw)

    @staticmethod
    def _batch(X, L):
        torch = _torch()
        if X.dtype != torch.bfloat16 or X.dim() != 2 or X.shape[1] != IN or not X.is_contiguous() or not X.is_cuda:
            raise PatchTableError(1, "X must be a contiguous CUDA bfloat16 [B x 16] tensor")
        if L.dtype != torch.uint8 or L.shape != (X.shape[0], 8) or not L.is_contiguous() or not L.is_cuda:
            raise PatchTableError(1, "labels must be a contiguous CUDA uint8 [B x 8] tensor")
        return X.shape[0], torch.cuda.current_stream().cuda_stream

    def train_step(self, X, L, lr: float, wd: float = 1e-4, want_loss: bool = False):
        """One AdamW step on a batch on torch's current stream; returns the mean loss if asked."""
        B, st = self._batch(X, L)
        loss = C.c_float()
        _check(lib().pt_proposal_train_step(self.handle, C.c_void_p(X.data_ptr()), C.c_void_p(L.data_ptr()), B,
                                            C.c_float(lr), C.c_float(wd), C.byref(loss) if want_loss else None,
                                            C.c_void_p(st)))
        return loss.value if want_loss else None

    def gradient(self, X, L):
        """(mean loss, FP32 gradient vector) of a batch, without updating."""
        B, st = self._batch(X, L)
        loss = C.c_float()
        g = np.empty(num_params(), np.float32)
        _check(lib().pt_proposal_gradient(self.handle, C.c_void_p(X.data_ptr()), C.c_void_p(L.data_ptr()), B,
                                          C.byref(loss), g.ctypes.data_as(C.c_void_p), C.c_void_p(st)))
        return loss.value, g

    def forward(self, X):
        torch = _torch()
        st = torch.cuda.current_stream().cuda_stream
        out = torch.empty((X.shape[0], OUT), dtype=torch.float32, device=X.device)
        _check(lib().pt_proposal_forward(self.handle, C.c_void_p(X.data_ptr()), X.shape[0], C.c_void_p(out.data_ptr()),
                                         C.c_void_p(st)))
        return out


def _srand(seed: int) -> None:
    C.CDLL(None).srand(C.c_uint(seed))


def samples_for_pair(a: np.ndarray, b: np.ndarray, switches: str = DEFAULT_SWITCHES, table: PatchTable | None = None):
    """(X, labels, ann) on the device for one pair: the plain lookup's NNF and its training samples."""
    torch = _torch()
    h, w = a.shape[:2]
    P = (h - 7) * (w - 7)
    if table is None:
        _srand(0)
        table = PatchTable(PatchTableParams(switches), b)
    st = torch.cuda.current_stream().cuda_stream
    a_d = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    ann = torch.empty(P * 3, dtype=torch.float64, device="cuda")
    table.lookup_device(a_d.data_ptr(), h, w, ann.data_ptr(), st)
    X = torch.empty((P, IN), dtype=torch.bfloat16, device="cuda")
    L = torch.empty((P, 8), dtype=torch.uint8, device="cuda")
    table.proposal_samples(a_d.data_ptr(), h, w, ann.data_ptr(), X.data_ptr(), L.data_ptr(), st)
    return X, L, ann


def collect(seeds, h: int, w: int, switches: str = DEFAULT_SWITCHES, per_pair: int | None = None, log=None):
    """Training samples of the plain method over seeded pairs (per_pair: random subset per pair)."""
    torch = _torch()
    Xs, Ls = [], []
    g = torch.Generator(device="cuda")
    g.manual_seed(12345)
    t0 = time.time()
    for i, seed in enumerate(seeds):
        a, b = synth.pair(h, w, seed)
        X, L, _ = samples_for_pair(a, b, switches)
        if per_pair and per_pair < X.shape[0]:
            idx = torch.randperm(X.shape[0], device="cuda", generator=g)[:per_pair]
            X, L = X.index_select(0, idx), L.index_select(0, idx)
        Xs.append(X)
        Ls.append(L)
        if log and (i % 20 == 0 or i == len(seeds) - 1):
            log("collect %d/%d pairs, %.1f s" % (i + 1, len(seeds), time.time() - t0))
    return torch.cat(Xs), torch.cat(Ls)


def label_stats(L) -> dict:
    """Fraction of samples whose match bin lies in the 5^G window, and per-dimension offset histogram."""
    Lc = L.cpu().numpy()
    used = Lc[:, :DIMS] != 0xFF
    off = np.where(used, Lc[:, :DIMS] & 7, -1)
    hist = [[int(((off[:, d] == k)).sum()) for k in range(CLASSES)] for d in range(DIMS)]
    return dict(samples=int(len(Lc)), exact_window=float(Lc[:, 6].mean()), offset_hist=hist)


def fit(net: ProposalNet, X, L, epochs: int = 4, batch: int = 8192, lr: float = 2e-3, wd: float = 1e-4,
        seed: int = 0, log=None):
    """AdamW over shuffled batches with a cosine learning-rate decay; returns the logged losses."""
    torch = _torch()
    N = (X.shape[0] // batch) * batch
    if N == 0:
        raise PatchTableError(1, "fewer samples (%d) than one batch (%d)" % (X.shape[0], batch))
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    steps = epochs * (N // batch)
    losses = []
    k = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(X.shape[0], device="cuda", generator=g)[:N]
        for i in range(N // batch):
            idx = perm[i * batch:(i + 1) * batch]
            xb, lb = X.index_select(0, idx), L.index_select(0, idx)
            cur = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * k / max(1, steps - 1))))
            want = (k % 200 == 0) or k == steps - 1
            loss = net.train_step(xb, lb, cur, wd, want_loss=want)
            if want:
                losses.append((k, loss))
                if log:
                    log("step %d/%d epoch %d loss %.4f lr %.2e (%.1f s)" % (k, steps, ep, loss, cur, time.time() - t0))
            k += 1
    _check(lib().pt_proposal_sync(net.handle, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return losses


def proposal_hits(table: PatchTable, net: ProposalNet, a: np.ndarray, ann) -> dict:
    """How often the plain method's match is among the proposals, overall and for confident patches."""
    torch = _torch()
    h, w = a.shape[:2]
    P = (h - 7) * (w - 7)
    st = torch.cuda.current_stream().cuda_stream
    a_d = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    cand = torch.empty((P, TOPK), dtype=torch.int32, device="cuda")
    conf = torch.empty(P, dtype=torch.float32, device="cuda")
    table.proposal_infer(net, a_d.data_ptr(), h, w, cand.data_ptr(), conf.data_ptr(), 0, st)
    A = ann.view(P, 3)
    mx, my = A[:, 0].to(torch.int32) + 7, A[:, 1].to(torch.int32) + 7
    key = mx | (my << 16)
    hit = (cand == key[:, None]).any(dim=1)
    c = conf >= net.threshold
    return dict(hit=float(hit.float().mean()), confident=float(c.float().mean()),
                hit_confident=float(hit[c].float().mean()) if bool(c.any()) else 0.0,
                mean_conf=float(conf.mean()))


EVAL_SCHEDULES = ((1, 1, 0), (1, 2, 1), (2, 2, 0), (3, 4, 0), (4, 8, 0))


def evaluate(net: ProposalNet, seeds, h: int, w: int, switches: str = DEFAULT_SWITCHES, schedules=EVAL_SCHEDULES,
             thresholds=(0.5, 0.0), log=None) -> dict:
    """Plain and learned queries on held-out pairs: per schedule (passes, first jump, pull
    candidates) the mean NNF distance (mean of sqrt) and the best device time of 3 lookups, averaged
    over the seeds, plus how often the plain match is among the proposals."""
    torch = _torch()
    from .metrics import get_mean_dist
    P = (h - 7) * (w - 7)
    st = torch.cuda.current_stream().cuda_stream
    acc = {}
    hits = []
    for seed in seeds:
        a, b = synth.pair(h, w, seed)
        _srand(0)
        params = PatchTableParams(switches)
        table = PatchTable(params, b)
        a_d = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
        ann = torch.empty(P * 3, dtype=torch.float64, device="cuda")
        params.gpu_prop_passes = 0
        table.lookup_device(a_d.data_ptr(), h, w, ann.data_ptr(), st)
        net.configure(0.5, False)
        hits.append(proposal_hits(table, net, a, ann))
        for sched in schedules:
            params.gpu_prop_passes, params.gpu_jump, params.gpu_pull_max = sched
            for kind in ("plain",) + tuple("learned_%g" % t for t in thresholds):
                best = None
                for rep in range(4):
                    if kind == "plain":
                        ms, _ = table.lookup_profile(a_d.data_ptr(), h, w, ann.data_ptr(), st)
                    else:
                        net.configure(float(kind.split("_")[1]), False)
                        ms, _ = table.lookup_learned_profile(net, a_d.data_ptr(), h, w, ann.data_ptr(), st)
                    if rep:
                        tot = sum(ms.values())
                        best = tot if best is None else min(best, tot)
                md = get_mean_dist(ann.view(h - 7, w - 7, 3).cpu().numpy())
                acc.setdefault("%d/%d/%d %s" % (sched + (kind,)), []).append((md, best))
        table.close()
        if log:
            log("evaluated seed %d" % seed)
    rows = {k: {"mean_nnf_dist": float(np.mean([m for m, _ in v])), "ms": float(np.mean([t for _, t in v])),
                "patches_per_s": P / (float(np.mean([t for _, t in v])) / 1000.0)} for k, v in acc.items()}
    hit = {k: float(np.mean([hh[k] for hh in hits])) for k in hits[0]}
    return {"size": [h, w], "seeds": list(seeds), "switches": switches, "proposal_hits": hit, "results": rows}


ABLATION_SCHEDULES = ((1, 2, 1), (1, 2, 0), (2, 2, 0), (3, 4, 0), (4, 8, 0))


def ablation(net: ProposalNet, seeds, h: int, w: int, switches: str = DEFAULT_SWITCHES, schedules=ABLATION_SCHEDULES,
             log=None) -> dict:
    """What a proposal network can gain at most, on held-out pairs.

    For every schedule, the mean NNF distance and the device time of: the plain query; the learned
    query with this network's proposals (threshold 0.5 and 0); and the learned query with *perfect*
    proposals -- each patch's own match in the plain method's converged (default-schedule) field,
    offered as its only proposal with confidence 1 -- timed without any inference cost.  The perfect
    proposals bound every network of this form: a network can at best reach their quality, and must
    add its inference time.  Two partial forms show how the gain falls with recall: perfect
    proposals only for patches whose match lies in the class space (bin offsets within the 5^G
    window the network scores), and only for a random subset as large as this network's recall.
    Also recorded: how often the converged match is among this network's 8 proposals (recall@8)
    and how often a label exists at all, with labels taken from the converged field and from a
    one-pass field."""
    torch = _torch()
    from .metrics import get_mean_dist
    P = (h - 7) * (w - 7)
    st = torch.cuda.current_stream().cuda_stream
    acc, hits, windows, inf_ms = {}, [], {"converged": [], "one_pass": []}, []

    def best_of(fn, reps=4):
        best = None
        for r in range(reps):
            ms, _ = fn()
            if r:
                tot = sum(ms.values())
                best = tot if best is None else min(best, tot)
        return best

    for seed in seeds:
        a, b = synth.pair(h, w, seed)
        _srand(0)
        params = PatchTableParams(switches)
        table = PatchTable(params, b)
        a_d = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
        ann = torch.empty(P * 3, dtype=torch.float64, device="cuda")
        params.gpu_prop_passes = 0
        table.lookup_device(a_d.data_ptr(), h, w, ann.data_ptr(), st)
        conv = ann.clone()
        # perfect proposals: the converged match (packed padded position) in slot 0, confidence 1
        A = conv.view(P, 3)
        perfect = torch.full((P, TOPK), -1, dtype=torch.int32, device="cuda")
        perfect[:, 0] = (A[:, 0].to(torch.int32) + 7) | ((A[:, 1].to(torch.int32) + 7) << 16)
        ones = torch.ones(P, dtype=torch.float32, device="cuda")
        net.configure(0.5, False)
        hits.append(proposal_hits(table, net, a, conv))
        X = torch.empty((P, IN), dtype=torch.bfloat16, device="cuda")
        L = torch.empty((P, 8), dtype=torch.uint8, device="cuda")
        table.proposal_samples(a_d.data_ptr(), h, w, conv.data_ptr(), X.data_ptr(), L.data_ptr(), st)
        windows["converged"].append(label_stats(L)["exact_window"])
        # perfect proposals for the patches a network of this class space could name at all (the
        # match's bin offsets inside the window), and for a random subset the size of this
        # network's recall: the other patches keep the plain candidates
        in_window = (L[:, 6] != 0).to(torch.float32)
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        at_recall = (torch.rand(P, device="cuda", generator=g) < hits[-1]["hit"]).to(torch.float32)
        params.gpu_prop_passes, params.gpu_jump, params.gpu_pull_max = 1, 2, 1
        table.lookup_device(a_d.data_ptr(), h, w, ann.data_ptr(), st)
        table.proposal_samples(a_d.data_ptr(), h, w, ann.data_ptr(), X.data_ptr(), L.data_ptr(), st)
        windows["one_pass"].append(label_stats(L)["exact_window"])
        cand = torch.empty((P, TOPK), dtype=torch.int32, device="cuda")
        conf = torch.empty(P, dtype=torch.float32, device="cuda")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = None
        for r in range(4):
            e0.record()
            table.proposal_infer(net, a_d.data_ptr(), h, w, cand.data_ptr(), conf.data_ptr(), 0, st)
            e1.record()
            e1.synchronize()
            if r:
                best = e0.elapsed_time(e1) if best is None else min(best, e0.elapsed_time(e1))
        inf_ms.append(best)
        for sched in schedules:
            params.gpu_prop_passes, params.gpu_jump, params.gpu_pull_max = sched
            arms = {"plain": lambda: table.lookup_profile(a_d.data_ptr(), h, w, ann.data_ptr(), st)}
            for name, cf in (("perfect_proposals", ones), ("perfect_in_window", in_window), ("perfect_at_net_recall", at_recall)):
                arms[name] = (lambda c_=cf: table.lookup_proposed_profile(
                    a_d.data_ptr(), h, w, perfect.data_ptr(), c_.data_ptr(), 0.5, ann.data_ptr(), st))
            for thr in (0.5, 0.0):
                arms["network_%g" % thr] = (lambda t_=thr: (net.configure(t_, False), table.lookup_learned_profile(
                    net, a_d.data_ptr(), h, w, ann.data_ptr(), st))[1])
            for kind, fn in arms.items():
                ms = best_of(fn)
                md = get_mean_dist(ann.view(h - 7, w - 7, 3).cpu().numpy())
                acc.setdefault("%d/%d/%d %s" % (sched + (kind,)), []).append((md, ms))
        table.close()
        if log:
            log("ablation seed %d" % seed)
    rows = {k: {"mean_nnf_dist": float(np.mean([m for m, _ in v])), "ms": float(np.mean([t for _, t in v]))}
            for k, v in acc.items()}
    return {"size": [h, w], "seeds": list(seeds), "switches": switches,
            "inference_ms": float(np.mean(inf_ms)),
            "recall_at_8": {k: float(np.mean([hh[k] for hh in hits])) for k in hits[0]},
            "label_in_window": {k: float(np.mean(v)) for k, v in windows.items()},
            "results": rows}


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--pairs", type=int, default=200)
    t.add_argument("--size", default="240x320", help="HxW of the training pairs")
    t.add_argument("--per-pair", type=int, default=0)
    t.add_argument("--epochs", type=int, default=4)
    t.add_argument("--batch", type=int, default=8192)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--switches", default=DEFAULT_SWITCHES)
    t.add_argument("--out", required=True)
    t.add_argument("--seed", type=int, default=0)
    e = sub.add_parser("eval")
    e.add_argument("--weights", required=True)
    e.add_argument("--heldout", type=int, default=20)
    e.add_argument("--size", default="1080x1920")
    e.add_argument("--switches", default=DEFAULT_SWITCHES)
    e.add_argument("--out", required=True)
    b = sub.add_parser("ablation")
    b.add_argument("--weights", required=True)
    b.add_argument("--heldout", type=int, default=5)
    b.add_argument("--size", default="1080x1920")
    b.add_argument("--switches", default=DEFAULT_SWITCHES)
    b.add_argument("--out", required=True)
    args = ap.parse_args()
    if args.cmd == "ablation":
        h, w = (int(v) for v in args.size.split("x"))
        net = ProposalNet.load(args.weights)
        res = ablation(net, HELDOUT_SEEDS[:args.heldout], h, w, args.switches, log=lambda m: print(m, flush=True))
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1, sort_keys=True)
        print(json.dumps({k: res[k] for k in ("inference_ms", "recall_at_8", "label_in_window")}))
        return
    if args.cmd == "eval":
        h, w = (int(v) for v in args.size.split("x"))
        net = ProposalNet.load(args.weights)
        res = evaluate(net, HELDOUT_SEEDS[:args.heldout], h, w, args.switches, log=lambda m: print(m, flush=True))
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1, sort_keys=True)
        print(json.dumps(res["proposal_hits"]))
        return
    if args.cmd == "train":
        h, w = (int(v) for v in args.size.split("x"))
        log = lambda m: print(m, flush=True)
        X, L = collect(TRAIN_SEEDS[:args.pairs], h, w, args.switches, args.per_pair or None, log)
        log("labels: %s" % json.dumps(label_stats(L)))
        net = ProposalNet(seed=args.seed)
        fit(net, X, L, args.epochs, args.batch, args.lr, log=log)
        net.save(args.out)
        log("saved %s" % args.out)


if __name__ == "__main__":
    _main()
