"""Generates wh_tables.h: the 8x8 Walsh-Hadamard masks of the reference's Gray-code kernels as
separable sign vectors, for the direct (sliding-window) descriptor kernel.

The reference computes kernel i >= 1 from kernel i-1 by the snake-order recurrence
``out_i(p) = s*out_i(p - d) + out_{i-1}(p) + s*out_{i-1}(p - d)`` (patchtable/gck.h:215-1950,
generated by patchtable/gck.py:360-420), starting from the 8x8 box (gck.h:52-205).  Running that
recurrence in exact integer arithmetic on an impulse image yields each kernel's mask M_i, with
response(y, x) = sum_{a,b} M_i[a][b] * in(y - 7 + a, x - 7 + b); every M_i is an outer product
V_i[a] * H_i[b] of +-1 vectors, which is what the CUDA kernel evaluates.

Run:  python patchtable_b200/csrc/gen_wh_tables.py
"""
import math
import os

import numpy as np


def _snake_order(w):
    cells = [(r, c) for r in range(w) for c in range(w)]

    def key(rc):
        r, c = rc
        m = max(r, c)
        return m + 0.5 + (r - c + w) * (1.0 / (4 * w)) * (-1 if m % 2 == 0 else 1)
    return sorted(cells, key=key)


def _alpha(w):
    k = int(round(math.log(w, 2)))
    out, sign_level = [], [1] * k

    def rec(n, level, a):
        a1, a2 = a + [sign_level[level]], a + [-sign_level[level]]
        sign_level[level] = -sign_level[level]
        if n * 2 == w:
            out.extend([a1, a2])
        else:
            rec(n * 2, level + 1, a1)
            rec(n * 2, level + 1, a2)
    rec(1, 0, [])
    return out


def recurrence_steps(w=8):
    order, alpha = _snake_order(w), _alpha(w)
    steps = []
    for i in range(1, w * w):
        horiz = order[i][1] != order[i - 1][1]
        j = 1 if horiz else 0
        a1, a2 = alpha[order[i - 1][j]], alpha[order[i][j]]
        idx = [a1[t] != a2[t] for t in range(len(a1))].index(True)
        steps.append((horiz, 2 ** idx, a2[idx]))
    return steps


def masks(n=64):
    """Mask of kernels 0..n-1 by simulating the recurrence on an impulse."""
    S = 40
    img = np.zeros((S, S), np.int64)
    py = px = 16
    img[py, px] = 1
    # kernel 0: full 8x8 box, response(y, x) = sum in(y-7..y, x-7..x)
    k0 = np.zeros((S, S), np.int64)
    for y in range(S):
        for x in range(S):
            k0[y, x] = img[max(0, y - 7):y + 1, max(0, x - 7):x + 1].sum()
    outs = [k0]
    for (horiz, d, s) in recurrence_steps()[:n - 1]:
        prev = outs[-1]
        cur = np.zeros_like(prev)
        for y in range(S):
            for x in range(S):
                yp, xp = (y, x - d) if horiz else (y - d, x)
                z = (lambda a: a[yp, xp] if (0 <= yp < S and 0 <= xp < S) else 0)
                cur[y, x] = s * z(cur) + prev[y, x] + s * z(prev)
        outs.append(cur)
    res = []
    for K in outs:
        M = np.zeros((8, 8), np.int64)
        for a in range(8):
            for b in range(8):
                M[a, b] = K[py + 7 - a, px + 7 - b]
        assert np.abs(K).sum() == 64, "response must be confined to the 8x8 window"
        V = M[:, 0] * M[0, 0]
        H = M[0, :]
        assert np.array_equal(np.outer(V, H), M)
        res.append((V, H))
    return res


def main():
    ms = masks(64)
    lines = ["/* Generated by gen_wh_tables.py; do not edit.  Mask of Gray-code kernel i is",
             "   M_i[a][b] = PT_WH_V[i][a] * PT_WH_H[i][b] over the patch rows a and columns b. */",
             "#pragma once", "static const signed char PT_WH_V[64][8] = {"]
    lines += ["    {%s}," % ", ".join(str(int(v)) for v in V) for V, _ in ms]
    lines += ["};", "static const signed char PT_WH_H[64][8] = {"]
    lines += ["    {%s}," % ", ".join(str(int(v)) for v in H) for _, H in ms]
    lines += ["};", ""]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "wh_tables.h")
    with open(path, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
