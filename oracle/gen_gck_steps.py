"""Generates oracle/gck_steps.h: the per-kernel recurrence steps of the reference's Gray-code
kernels (test infrastructure).

Restates patchtable/gck.py:37-82 (snake order, Walsh-Hadamard basis in Gray-code sequence,
delta/sign of each step) and patchtable/gck.py:360-420 (how each kernel i >= 1 is computed from
kernel i-1 by ``out_i(p) = s*out_i(p - d) + out_{i-1}(p) + s*out_{i-1}(p - d)`` with d a
horizontal or vertical shift of 2**idx).  The known answers of gck.py:69-79 are checked on import.

Run:  python oracle/gen_gck_steps.py   (rewrites oracle/gck_steps.h)
"""
import math
import os


def snake_order(w):
    """gck.py:37-39: cells (row, col) sorted along the anti-diagonal snake."""
    cells = [(r, c) for r in range(w) for c in range(w)]

    def key(rc):
        r, c = rc
        m = max(r, c)
        return m + 0.5 + (r - c + w) * (1.0 / (4 * w)) * (-1 if m % 2 == 0 else 1)
    return sorted(cells, key=key)


def wh_basis(w, alpha=False):
    """gck.py:46-67: Walsh-Hadamard vectors of length w in Gray-code order (or their alpha
    sign sequences)."""
    k = int(round(math.log(w, 2)))
    out = []
    sign_level = [1] * k

    def rec(vec, level, alpha_vec):
        v1 = vec + [sign_level[level] * x for x in vec]
        v2 = vec + [-sign_level[level] * x for x in vec]
        a1 = alpha_vec + [sign_level[level]]
        a2 = alpha_vec + [-sign_level[level]]
        sign_level[level] = -sign_level[level]
        if len(v1) == w:
            out.extend([a1, a2] if alpha else [v1, v2])
        else:
            rec(v1, level + 1, a1)
            rec(v2, level + 1, a2)
    rec([1], 0, [])
    return out


def delta_and_sign(a1, a2):
    """gck.py:41-44."""
    idx = [a1[i] != a2[i] for i in range(len(a1))].index(True)
    return 2 ** idx, a1[idx], a2[idx]


def steps(w=8):
    """[(horizontal, delta, sign)] for kernels 1 .. w*w-1 (gck.py:364-378)."""
    order = snake_order(w)
    alpha = wh_basis(w, alpha=True)
    out = []
    for i in range(1, len(order)):
        horiz = order[i][1] != order[i - 1][1]
        if horiz:
            d, s1, s2 = delta_and_sign(alpha[order[i - 1][1]], alpha[order[i][1]])
        else:
            d, s1, s2 = delta_and_sign(alpha[order[i - 1][0]], alpha[order[i][0]])
        assert {s1, s2} == {-1, 1}
        out.append((int(horiz), d, s2))
    return out


def _known_answers():
    """gck.py:69-79."""
    assert wh_basis(4) == [[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]]
    assert wh_basis(8) == [[1, 1, 1, 1, 1, 1, 1, 1], [1, 1, 1, 1, -1, -1, -1, -1],
                           [1, 1, -1, -1, -1, -1, 1, 1], [1, 1, -1, -1, 1, 1, -1, -1],
                           [1, -1, -1, 1, 1, -1, -1, 1], [1, -1, -1, 1, -1, 1, 1, -1],
                           [1, -1, 1, -1, -1, 1, -1, 1], [1, -1, 1, -1, 1, -1, 1, -1]]
    assert wh_basis(4, alpha=True) == [[1, 1], [1, -1], [-1, -1], [-1, 1]]
    assert wh_basis(8, alpha=True) == [[1, 1, 1], [1, 1, -1], [1, -1, -1], [1, -1, 1],
                                       [-1, -1, 1], [-1, -1, -1], [-1, 1, -1], [-1, 1, 1]]


_known_answers()


def main():
    st = steps(8)
    lines = ["/* Generated by oracle/gen_gck_steps.py from the restated gck.py snake order; do not edit.",
             "   Step i (kernel i+1) : {horizontal, delta, sign}. */",
             "#ifndef PT_ORACLE_GCK_STEPS_H", "#define PT_ORACLE_GCK_STEPS_H",
             "static const int ORC_GCK_STEPS[63][3] = {"]
    lines += ["    {%d, %d, %d}," % s for s in st]
    lines += ["};", "#endif", ""]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gck_steps.h")
    with open(path, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
