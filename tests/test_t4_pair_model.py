"""CPU model of the paired type-4 steps (the element-wise line steps
Op_t4_pre / Op_t4_post in minfft_b200/csrc/line_ops.cuh, and the same
algebra in the fused chain stages LoadT4Chain / StoreT4Chain of
minfft_b200/csrc/axis_pass.cuh), checked against the double-precision oracle.

A DCT-4 / DST-4 of N reals runs a complex DFT of L = N/2 points.  Each item of
the pre-rotation takes the point n < L/2 with its mirror n' = L-1-n: it reads
the reals (x[2n], x[2n+1]) and (x[N-2-2n], x[N-1-2n]) and writes
z[n] = w_2N^n (x[2n] + i x[N-1-2n]) and z[n'] = w_2N^n' (x[N-2-2n] + i x[2n+1])
(conjugated and negated for the DST-4).  Each item of the post-rotation takes
the spectrum values T_m and U = T_(L-1-m) and writes y[2m], y[2m+1],
y[N-2-2m], y[N-1-2m] as 2 Re (2 Im for the DST-4) of g_k times T_m, conj(U),
U, conj(T_m), with g_k = w_8N^(2k+1).  The model follows those index
formulas literally (reference: minfft.c:891-975, s_dct4_1d / s_dst4_1d,
which form the same half-length DFT point by point); a slip in a mirror index shows up
as an O(1) error against the oracle."""
import numpy as np
import pytest

import oracle
from conftest import rel_l2


def w(m, e):
    return np.exp(-2j * np.pi * np.asarray(e, dtype=np.float64) / m)


def t4_pairs(x, dst):
    n_pts = x.size
    half = n_pts // 2
    n = np.arange(half // 2)
    mir = half - 1 - n
    x0, x1, y0, y1 = x[2 * n], x[2 * n + 1], x[n_pts - 2 - 2 * n], x[n_pts - 1 - 2 * n]

    def rot(root, a, b):
        return -(root * (a - 1j * b)) if dst else root * (a + 1j * b)

    z = np.empty(half, complex)
    z[n] = rot(w(2 * n_pts, n), x0, y1)
    z[mir] = rot(w(2 * n_pts, mir), y0, x1)
    t = np.fft.fft(z)

    def g(k):
        return w(8 * n_pts, 2 * np.asarray(k) + 1)

    def part(v):
        return 2 * (v.imag if dst else v.real)

    m = np.arange(half // 2)
    tm, u = t[m], t[half - 1 - m]
    y = np.empty(n_pts)
    y[2 * m] = part(g(2 * m) * tm)
    y[n_pts - 1 - 2 * m] = part(g(n_pts - 1 - 2 * m) * np.conj(tm))
    y[n_pts - 2 - 2 * m] = part(g(n_pts - 2 - 2 * m) * u)
    y[2 * m + 1] = part(g(2 * m + 1) * np.conj(u))
    return y


@pytest.mark.parametrize("n_pts", [16, 64, 1024, 1 << 14])
@pytest.mark.parametrize("op", ["dct4", "dst4"])
def test_paired_type4_steps_match_oracle(n_pts, op):
    rng = np.random.default_rng(n_pts)
    x = rng.uniform(-1, 1, n_pts)
    got = t4_pairs(x, op == "dst4")
    assert rel_l2(got, oracle.apply(op, x, (n_pts,), single=False)) <= 1e-13


def test_mirror_root_identity():
    """The fused store forms the mirror's root from its own:
    w_8N^(2N-1-4m) = -i conj(w_8N^(4m+1)) (StoreT4Chain)."""
    n_pts = 1 << 12
    m = np.arange(n_pts // 4)
    lhs = w(8 * n_pts, 2 * n_pts - 1 - 4 * m)
    rhs = -1j * np.conj(w(8 * n_pts, 4 * m + 1))
    assert np.max(np.abs(lhs - rhs)) <= 1e-14
