"""Learned proposal network: the library's features, labels, forward and backward kernels against
the CPU float64 oracle (oracle/proposal_ref.py), the fused inference kernel against the unfused
GEMM path, training, and the learned query's NNF.

Tolerances: features and label bytes are bit-exact (float32 arithmetic, then BF16 rounding).  The
GPU accumulates BF16 products in FP32 in a different order than the oracle's float64, and a
rounding to BF16 of an intermediate value can land one BF16 step apart; against the oracle that
rounds at the same points the gradient's relative L2 error per tensor must stay below 5e-3, and
below 5e-2 against the oracle without any BF16 rounding."""
import ctypes

import numpy as np
import pytest

import patchtable_b200 as ptb
from oracle import proposal_ref as R
from patchtable_b200 import synth

GRAD_RTOL_EMULATED = 5e-3
GRAD_RTOL_EXACT = 5e-2


def _rand_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    d = {"W1": rng.normal(0, 0.4, (R.HIDDEN, R.IN)), "b1": rng.normal(0, 0.1, R.HIDDEN),
         "W2": rng.normal(0, 0.12, (R.HIDDEN, R.HIDDEN)), "b2": rng.normal(0, 0.1, R.HIDDEN),
         "W3": rng.normal(0, 0.1 * scale, (R.OUT, R.HIDDEN)), "b3": rng.normal(0, 0.1, R.OUT)}
    d["W1"][:, 12:] = 0
    return R.pack(d)


def _rand_batch(seed, B):
    rng = np.random.default_rng(seed)
    X = np.zeros((B, R.IN))
    X[:, :12] = rng.uniform(-0.6, 0.6, (B, 12))
    X = R.bf16(X)
    L = np.zeros((B, 8), np.uint8)
    for d in range(R.DIMS):
        lo, hi = rng.integers(0, 3, B), rng.integers(0, 3, B)
        y = np.array([rng.integers(2 - l, 3 + h) for l, h in zip(lo, hi)])
        L[:, d] = y | (lo << 3) | (hi << 5)
    L[rng.random(B) < 0.05, 5] = 0xFF
    return X, L


# ---------------------------------------------------------------- CPU: the oracle itself


def test_bf16_rounding_known_values():
    v = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, 1 + 2 ** -7, -2.5, 3.0e38, 1e-40])
    r = R.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # tie -> even
    assert r[2] == 1 + 2 ** -6               # tie -> even (odd neighbour below)
    assert r[3] == 1 + 2 ** -7               # representable
    assert r[4] == -2.5
    assert np.isfinite(r[5])
    assert R.bf16_bits(np.array([1.0]))[0] == 0x3F80


def test_oracle_gradient_is_the_derivative_of_its_loss():
    """Central differences of the exact (no rounding) float64 loss."""
    params = _rand_params(3, scale=3.0)
    X, L = _rand_batch(4, 24)
    _, g = R.loss_and_grad(params, X, L, emulate=False)
    rng = np.random.default_rng(5)
    idx = rng.choice(len(params), 60, replace=False)
    for i in idx:
        e = np.zeros_like(params)
        e[i] = 1e-6
        lp, _ = R.loss_and_grad(params + e, X, L, emulate=False)
        lm, _ = R.loss_and_grad(params - e, X, L, emulate=False)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def _beam_topk(logits, bins, nslices, k=R.TOPK):
    """The search the inference kernel runs: keep the k best prefixes, dimension by dimension."""
    beam = [(0.0, ())]
    for d in range(len(nslices)):
        z = np.asarray(logits[d * 5:(d + 1) * 5], np.float64)
        ok = [0 <= bins[d] + o - 2 < nslices[d] for o in range(5)]
        m = max(z[o] for o in range(5) if ok[o])
        ls = m + np.log(sum(np.exp(z[o] - m) for o in range(5) if ok[o]))
        nxt = [(s + z[o] - ls, offs + (o - 2,)) for s, offs in beam for o in range(5) if ok[o]]
        nxt.sort(key=lambda t: -t[0])
        beam = nxt[:k]
    return beam


def test_beam_search_is_exact_top8():
    rng = np.random.default_rng(7)
    for _ in range(40):
        logits = rng.normal(0, 2, 32)
        nslices = [int(x) for x in rng.integers(1, 6, 6)]
        bins = [int(rng.integers(0, n)) for n in nslices]
        a = _beam_topk(logits, bins, nslices)
        b = R.topk_cells(logits, bins, nslices)
        assert len(a) == len(b)
        assert np.allclose([s for s, _ in a], [s for s, _ in b], atol=1e-12)


# ---------------------------------------------------------------- GPU


def _table_and_pair(libc, h=120, w=160, seed=11, sw="-speed 3 -coherence_spatial 4 -limit 2"):
    a, b = synth.pair(h, w, seed)
    libc.srand(1)
    t = ptb.PatchTable(ptb.PatchTableParams(sw), b)
    return t, a, b


def _parts(t):
    ns, _ = t.shape()
    return [t.partition(d) for d in range(len(ns))], ns


@pytest.mark.gpu
def test_samples_bit_exact(gpu, libc):
    import torch
    from patchtable_b200 import proposal as PR
    t, a, b = _table_and_pair(libc)
    X, L, ann = PR.samples_for_pair(a, b, table=t)
    torch.cuda.synchronize()
    parts, ns = _parts(t)
    h, w = a.shape[:2]
    qdesc = ptb.descriptor(t.params, a).reshape(-1, t.params.ndims)
    f, bins_a = R.features(qdesc, parts)
    got = X.view(torch.int16).cpu().numpy().view(np.uint16)
    assert np.array_equal(got, R.bf16_bits(f))
    A = ann.view(-1, 3).cpu().numpy()
    bdesc = t.descriptor().reshape(-1, t.params.ndims)
    bew = b.shape[1] - 7
    mi = A[:, 1].astype(np.int64) * bew + A[:, 0].astype(np.int64)
    _, bins_b = R.features(bdesc[mi], parts)
    want = R.labels(bins_a, bins_b, ns, np.ones(len(A), bool))
    assert np.array_equal(L.cpu().numpy(), want)


@pytest.mark.gpu
def test_gradient_matches_float64_oracle(gpu, libc):
    import torch
    from patchtable_b200 import proposal as PR
    t, a, b = _table_and_pair(libc, seed=12)
    X, L, _ = PR.samples_for_pair(a, b, table=t)
    B = 512
    X, L = X[:B].contiguous(), L[:B].contiguous()
    params = _rand_params(21, scale=4.0).astype(np.float32)
    net = PR.ProposalNet(params=params)
    loss, g = net.gradient(X, L)
    Xh = X.float().cpu().numpy().astype(np.float64)
    Lh = L.cpu().numpy()
    loss_e, g_e = R.loss_and_grad(params.astype(np.float64), Xh, Lh, emulate=True)
    loss_x, g_x = R.loss_and_grad(params.astype(np.float64), Xh, Lh, emulate=False)
    assert abs(loss - loss_e) <= 1e-4 * abs(loss_e)
    assert abs(loss - loss_x) <= 1e-2 * abs(loss_x)
    ge, gx, gg = R.unpack(g_e), R.unpack(g_x), R.unpack(g.astype(np.float64))
    for k in ge:
        n = np.linalg.norm(ge[k])
        assert n > 0
        assert np.linalg.norm(gg[k] - ge[k]) <= GRAD_RTOL_EMULATED * n, k
        assert np.linalg.norm(gg[k] - gx[k]) <= GRAD_RTOL_EXACT * np.linalg.norm(gx[k]), k


@pytest.mark.gpu
def test_fused_inference_matches_gemm_path_and_top8(gpu, libc):
    import torch
    from patchtable_b200 import proposal as PR
    t, a, b = _table_and_pair(libc, seed=13)
    X, L, _ = PR.samples_for_pair(a, b, table=t)
    params = _rand_params(31, scale=8.0).astype(np.float32)
    net = PR.ProposalNet(params=params)
    h, w = a.shape[:2]
    P = (h - 7) * (w - 7)
    a_d = torch.from_numpy(a).cuda()
    cand = torch.empty((P, 8), dtype=torch.int32, device="cuda")
    conf = torch.empty(P, dtype=torch.float32, device="cuda")
    logits = torch.empty((P, 32), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    t.proposal_infer(net, a_d.data_ptr(), h, w, cand.data_ptr(), conf.data_ptr(), logits.data_ptr(), st)
    ref = net.forward(X)
    torch.cuda.synchronize()
    assert torch.equal(logits, ref)               # same tensor-core products in the same order
    lo = logits.cpu().numpy().astype(np.float64)
    orc = R.forward(params.astype(np.float64), X.float().cpu().numpy().astype(np.float64), emulate=True)
    # a hidden activation rounded to the other BF16 neighbour moves a few logits by ~1e-2; the
    # rest agree to FP32 accumulation order
    assert np.linalg.norm(lo - orc) <= 1e-4 * np.linalg.norm(orc)
    assert np.mean(np.abs(lo - orc) <= 1e-4 * (1 + np.abs(orc))) >= 0.999
    parts, ns = _parts(t)
    qdesc = ptb.descriptor(t.params, a).reshape(-1, t.params.ndims)
    _, bins = R.features(qdesc, parts)
    table = t.table()
    strides = np.cumprod([1] + ns[::-1][:-1])[::-1]
    C, F = cand.cpu().numpy(), conf.cpu().numpy()
    rng = np.random.default_rng(0)
    checked = 0
    for p in rng.choice(P, 150, replace=False):
        top = R.topk_cells(lo[p], bins[p], ns, k=9)
        scores = [s for s, _ in top]
        assert abs(F[p] - np.exp(scores[0])) <= 1e-5
        if any(abs(scores[i] - scores[i + 1]) < 1e-4 for i in range(len(scores) - 1)):
            continue                              # near-tie: order may legitimately differ
        cells = [int(np.dot(bins[p] + np.array(o), strides)) for _, o in top[:8]]
        want = [int(table[c]) for c in cells] + [-1] * (8 - len(cells))
        assert list(C[p]) == want, p
        checked += 1
    assert checked >= 100


@pytest.mark.gpu
def test_training_reduces_loss(gpu, libc):
    from patchtable_b200 import proposal as PR
    X, L = PR.collect(PR.TRAIN_SEEDS[:4], 96, 128, "-speed 3 -coherence_spatial 4 -limit 2")
    net = PR.ProposalNet(seed=1)
    l0, _ = net.gradient(X[:4096].contiguous(), L[:4096].contiguous())
    losses = PR.fit(net, X, L, epochs=6, batch=1024, lr=3e-3)
    l1, _ = net.gradient(X[:4096].contiguous(), L[:4096].contiguous())
    assert np.isfinite(l1) and l1 < 0.8 * l0, (l0, l1, losses)


@pytest.mark.gpu
def test_learned_lookup_distances_exact(gpu, libc):
    from oracle.oracle import recompute_dists
    from patchtable_b200 import proposal as PR
    t, a, b = _table_and_pair(libc, h=96, w=128, seed=14)
    net = PR.ProposalNet(params=_rand_params(41, scale=8.0).astype(np.float32), threshold=0.0)
    ann = t.lookup_learned(a, net)
    assert np.all(ann[..., 0] >= 0) and np.all(ann[..., 0] < b.shape[1] - 7)
    assert np.all(ann[..., 1] >= 0) and np.all(ann[..., 1] < b.shape[0] - 7)
    rd = recompute_dists(a, b, ann)
    assert np.all(np.abs(ann[..., 2] - rd) <= 1e-5 * np.maximum(rd, 1e-12) + 1e-9)
    plain = t.lookup(a)
    # every patch scores its own stored match first, so both results stay within a few percent
    assert ann[..., 2].mean() <= 1.25 * plain[..., 2].mean()


@pytest.mark.gpu
def test_learned_threshold_one_is_plain(gpu, libc):
    """A threshold no patch reaches leaves every patch on the plain candidates."""
    from patchtable_b200 import proposal as PR
    t, a, b = _table_and_pair(libc, h=96, w=128, seed=15)
    net = PR.ProposalNet(seed=3, threshold=1.0)
    plain = t.lookup(a)
    learned = t.lookup_learned(a, net)
    assert np.array_equal(plain, learned)


WEIGHTS = "patchtable_b200/data/proposal_weights.npy"


@pytest.mark.gpu
def test_trained_network_gains_over_plain(gpu, libc):
    """The committed network (trained on the plain method's NNFs of pairs 5000-5199) on a held-out
    pair: with its proposals for every patch, one propagation pass reaches a lower mean NNF
    distance than the plain query with the same pass, every distance still exact."""
    import os
    from oracle.oracle import recompute_dists
    from patchtable_b200 import proposal as PR
    from patchtable_b200.metrics import get_mean_dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    net = PR.ProposalNet.load(os.path.join(root, WEIGHTS), threshold=0.0)
    a, b = synth.pair(540, 960, PR.HELDOUT_SEEDS[0])
    libc.srand(1)
    p = ptb.PatchTableParams(PR.DEFAULT_SWITCHES)
    t = ptb.PatchTable(p, b)
    p.gpu_prop_passes, p.gpu_jump, p.gpu_pull_max = 1, 1, 0
    plain = t.lookup(a)
    learned = t.lookup_learned(a, net)
    mp, ml = get_mean_dist(plain), get_mean_dist(learned)
    assert ml <= 0.98 * mp, (ml, mp)
    rd = recompute_dists(a, b, learned)
    assert np.all(np.abs(learned[..., 2] - rd) <= 1e-5 * np.maximum(rd, 1e-12) + 1e-9)
