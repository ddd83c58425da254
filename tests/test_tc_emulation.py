"""CPU model of the tensor-core split-precision arithmetic (the scheme the
kernel in minfft_b200/csrc/tc_pass.cu runs on tcgen05), checked against the
double-precision oracle.

Each 256-point transform is scaled by one power of two so that the largest
component of its input lies in [256, 512).  Per radix-16 stage, each row of
16 complex values is split into 16-bit terms (FP16: two, BF16: three) and
multiplied by the split real 32 x 32 form of the 16-point DFT matrix, keeping
the products Ai Bj with i + j < terms; the leading product and the
corrections accumulate in FP32 separately and are added; the stage-1 result is
twiddled in FP32, and the scale is undone at the end.  A Stockham chain of
two such passes over a 65536-point axis, the second pre-twiddled in FP32 with
roots built from table roots and their products as the kernel builds them, is
modelled too.  The model shows the scheme itself meets the 1e-6 relative-L2
bar with margin, so the GPU tests measure the kernel, not the method."""
import numpy as np
import pytest

import oracle
from conftest import rel_l2

F32 = np.float32


def to16(r, fmt):
    """Round FP32 values to FP16 or BF16 (nearest even), returned as FP32."""
    if fmt == "f16":
        return r.astype(np.float16).astype(F32)
    b = r.astype(F32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(F32)


def split(v, fmt):
    terms, r = [], v.astype(F32)
    for _ in range(2 if fmt == "f16" else 3):
        h = to16(r, fmt)
        terms.append(h)
        r = (r - h).astype(F32)
    return terms


def dft16_real():
    m = (np.arange(16)[:, None] * np.arange(16)[None, :]) % 16
    c = np.cos(2 * np.pi * m / 16)
    s = np.sin(2 * np.pi * m / 16)
    c[m % 8 == 4] = 0
    s[m % 8 == 0] = 0
    return np.block([[c, s], [-s, c]]).astype(F32)


def stage(rows, fmt):
    a = np.concatenate([rows.real, rows.imag], axis=1).astype(F32)
    at, bt = split(a, fmt), split(dft16_real(), fmt)
    lead = (at[0].astype(np.float64) @ bt[0].T.astype(np.float64)).astype(F32)
    corr = np.zeros((a.shape[0], 32), F32)
    for i in range(len(at)):
        for j in range(len(at) - i):
            if i + j:
                corr = (corr + (at[i].astype(np.float64) @ bt[j].T.astype(np.float64)).astype(F32)).astype(F32)
    d = (lead + corr).astype(F32)
    return (d[:, :16] + 1j * d[:, 16:]).astype(np.complex64)


def tc256(x, fmt):
    t = x.shape[0]
    x = x.astype(np.complex64)
    mx = np.maximum(np.abs(x.real), np.abs(x.imag)).max(axis=1).astype(F32)
    ex = ((mx.view(np.uint32) >> 23) & 0xFF).astype(np.int64)
    s = np.clip(135 - ex, -126, 126)
    sc = np.ldexp(np.ones(t), s).astype(F32)[:, None]
    v = (x * sc).astype(np.complex64).reshape(t, 16, 16)            # [t, n1, n2]
    y = stage(v.transpose(0, 2, 1).reshape(t * 16, 16), fmt).reshape(t, 16, 16)  # [t, n2, k1]
    tw = np.exp(-2j * np.pi * np.outer(np.arange(16), np.arange(16)) / 256).astype(np.complex64)
    y = (y * tw[None]).astype(np.complex64)
    z = stage(y.transpose(0, 2, 1).reshape(t * 16, 16), fmt).reshape(t, 16, 16)  # [t, k1, k2]
    return (z.transpose(0, 2, 1).reshape(t, 256) / sc).astype(np.complex64)


@pytest.mark.parametrize("fmt", ["f16", "bf16"])
@pytest.mark.parametrize("spread", [0.0, 20.0])
def test_split_scheme_meets_the_bar(fmt, spread):
    rng = np.random.default_rng(5)
    x = rng.standard_normal((64, 256)) + 1j * rng.standard_normal((64, 256))
    x *= np.exp(rng.uniform(-spread, spread, (64, 1)))
    got = tc256(x, fmt)
    for i in range(x.shape[0]):
        ref = oracle.apply("dft", x[i].astype(np.complex128), (256,), single=False, kind=oracle.best_kind())
        assert rel_l2(got[i], ref) <= 3e-7, (fmt, i)


def stockham_roots(lt):
    """w_lt^g for every g < lt as the kernel forms it: the product, in FP32,
    of a coarse root w_lt^(a << lo) and a fine root w_lt^c (c < 2^lo), both
    correctly rounded to FP32."""
    lo = (int(np.log2(lt)) + 1) // 2
    w = lambda e: np.exp(-2j * np.pi * e / lt).astype(np.complex64)  # noqa: E731
    g = np.arange(lt)
    return (w((g >> lo) << lo) * w(g & ((1 << lo) - 1))).astype(np.complex64)


def pretwiddles(lt, q):
    """Pre-twiddles w_lt^(q*n), n < 256, of the sub-DFTs with span index q in
    the second pass of a 256 x 256 chain, built as the tensor-core kernel
    builds them in column mode: element n = n0 + 16 i of a thread takes
    base * d4^(i >> 2) * d^(i & 3) with base = w^(n0 q), d = w^(16 q),
    d4 = w^(64 q) table roots and d^2, d^3, d^8, d^12 as FP32 products."""
    r = stockham_roots(lt)
    out = np.empty((len(q), 256), np.complex64)
    for n0 in range(16):
        base, d1, d4 = r[(n0 * q) % lt], r[(16 * q) % lt], r[(64 * q) % lt]
        d2 = (d1 * d1).astype(np.complex64)
        pw = [np.ones_like(d1), d1, d2, (d2 * d1).astype(np.complex64)]
        d8 = (d4 * d4).astype(np.complex64)
        pw4 = [None, d4, d8, (d8 * d4).astype(np.complex64)]
        for i in range(16):
            w = base
            if i >> 2:
                w = (w * pw4[i >> 2]).astype(np.complex64)
            if i & 3:
                w = (w * pw[i & 3]).astype(np.complex64)
            out[:, n0 + 16 * i] = w
    return out


@pytest.mark.parametrize("fmt", ["f16", "bf16"])
def test_split_scheme_in_a_stockham_chain_meets_the_bar(fmt):
    """A 65536-point DFT as the tensor-core mode plans it: two 256-point
    passes, x[n + 256 m] -> Y[n, q] (DFT over m) -> pre-twiddle w^(q n) in
    FP32 -> X[q + 256 k] (DFT over n), both passes in the split scheme."""
    lt = 1 << 16
    rng = np.random.default_rng(8)
    x = rng.standard_normal(lt) + 1j * rng.standard_normal(lt)
    a = x.astype(np.complex64).reshape(256, 256)          # a[m, n] = x[n + 256 m]
    y = tc256(np.ascontiguousarray(a.T), fmt)              # y[n, q]
    q = np.arange(256)
    yt = (y.T * pretwiddles(lt, q)).astype(np.complex64)  # yt[q, n]
    z = tc256(yt, fmt)                                     # z[q, k] = X[q + 256 k]
    got = z.T.reshape(lt)
    ref = oracle.apply("dft", x.astype(np.complex128), (lt,), single=False, kind=oracle.best_kind())
    assert rel_l2(got, ref) <= 5e-7, fmt


def test_chain_pretwiddles_match_exact_roots():
    """Each product-built pre-twiddle comes from six table roots and nine
    FP32 products at most: measured 7.2 * 2^-24 worst case and 1.6 * 2^-24
    RMS from the exact root, the size of the FP32 rounding of the data it
    multiplies."""
    lt = 1 << 16
    q = np.arange(256)
    got = pretwiddles(lt, q).astype(np.complex128)
    ref = np.exp(-2j * np.pi * np.outer(q, np.arange(256)) / lt)
    err = np.abs(got - ref)
    assert err.max() <= 12 * 2.0 ** -24
    assert np.sqrt(np.mean(err ** 2)) <= 2 * 2.0 ** -24


def test_split_terms_reconstruct_fp32():
    """Rows scaled into [256, 512): FP16 pairs keep 2^-22 of the row maximum
    (FP16's subnormal floor bounds the small elements), BF16 triples keep
    every element to 2^-23 of itself."""
    rng = np.random.default_rng(6)
    v = (rng.standard_normal(10000) * 100).astype(F32)
    v = np.clip(v, -511, 511).astype(F32)
    s = sum(t.astype(np.float64) for t in split(v, "f16"))
    assert np.max(np.abs(s - v)) <= 2.0 ** -22 * 256
    s = sum(t.astype(np.float64) for t in split(v, "bf16"))
    assert np.max(np.abs(s - v) / np.abs(v)) <= 2.0 ** -23
