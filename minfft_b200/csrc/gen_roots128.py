"""Writes roots128.h: w_128^m = exp(-2*pi*i*m/128) for m = 0..31, each part
correctly rounded to double and to float (the 128th roots of unity that the
axis-pass load and store stages multiply their per-thread table roots by).

The values are computed with Python's decimal module at 60 significant
digits (pi by Machin's formula, cos and sin by their Taylor series on the
exact angle), then rounded once to the target format, so no value carries a
double rounding.  Run from this directory: python gen_roots128.py
"""
import struct
from decimal import Decimal, getcontext

getcontext().prec = 60
COUNT = 32


def arctan_inv(x: int) -> Decimal:
    """arctan(1/x) by its Taylor series."""
    x = Decimal(x)
    term = 1 / x
    total = term
    x2 = x * x
    n = 1
    while True:
        term = -term / x2
        n += 2
        t = term / n
        if abs(t) < Decimal(10) ** -70:
            return total
        total += t


PI = 4 * (4 * arctan_inv(5) - arctan_inv(239))


def cos_sin(a: Decimal):
    c, s = Decimal(0), Decimal(0)
    term = Decimal(1)  # a^n / n!
    n = 0
    while abs(term) > Decimal(10) ** -70:
        if n % 4 == 0:
            c += term
        elif n % 4 == 1:
            s += term
        elif n % 4 == 2:
            c -= term
        else:
            s -= term
        n += 1
        term = term * a / n
    return c, s


def to_double(d: Decimal) -> float:
    return float(d)  # correctly rounded (decimal string to binary64)


def to_float(d: Decimal) -> float:
    """d rounded to the nearest binary32 (ties to even), exactly."""
    if d == 0:
        return 0.0
    if d < 0:
        return -to_float(-d)
    f = struct.unpack("f", struct.pack("f", float(d)))[0]
    best = None
    bits = struct.unpack("I", struct.pack("f", f))[0]
    for b in (bits - 1, bits, bits + 1):
        cand = struct.unpack("f", struct.pack("I", b & 0xFFFFFFFF))[0]
        err = abs(Decimal(cand) - d)
        if best is None or err < best[0] or (err == best[0] and (b & 1) == 0):
            best = (err, cand)
    return best[1]


def fmt_double(v: float) -> str:
    return "0.0" if v == 0 else float.hex(v)


def fmt_float(v: float) -> str:
    return "0.0f" if v == 0 else float.hex(v) + "f"  # the binary32 value, written exactly


def render() -> str:
    """Text of roots128.h."""
    re_d, im_d, re_f, im_f = [], [], [], []
    for m in range(COUNT):
        a = 2 * PI * m / 128
        c, s = cos_sin(a)
        re_d.append(fmt_double(to_double(c)))
        im_d.append(fmt_double(to_double(-s)))
        re_f.append(fmt_float(to_float(c)))
        im_f.append(fmt_float(to_float(-s)))

    def rows(vals):
        return ",\n".join("    " + ", ".join(vals[i:i + 4]) for i in range(0, len(vals), 4))

    out = f"""// Generated by gen_roots128.py -- do not edit.
// w_128^m = exp(-2*pi*i*m/128) = (cos, -sin)(2*pi*m/128), m = 0..{COUNT - 1},
// each part correctly rounded to double and to float.  Constant memory with
// static initialisers (internal linkage: every translation unit that includes
// this header holds its own copy, loaded with the module), so a loop index
// known after unrolling becomes a constant-bank operand.
#pragma once

namespace mb {{
namespace roots128 {{

constexpr int kCount = {COUNT};
static __constant__ double kReD[kCount] = {{
{rows(re_d)}}};
static __constant__ double kImD[kCount] = {{
{rows(im_d)}}};
static __constant__ float kReF[kCount] = {{
{rows(re_f)}}};
static __constant__ float kImF[kCount] = {{
{rows(im_f)}}};

}}  // namespace roots128
}}  // namespace mb
"""
    return out


if __name__ == "__main__":
    with open("roots128.h", "w") as f:
        f.write(render())
