"""Generate the golden vectors the oracle and the GPU engine are pinned to.

Run in a container where the reference sources are present:

    make -C oracle ref && python tests/golden/make_golden.py

It runs the reference library itself (aimukhin/minfft minfft.c, compiled
unmodified by oracle/Makefile into oracle/_ref/) on seeded inputs for every
transform and a spread of shapes -- the N = 1, 2, 4, 8 codelet sizes, the
first tabulated size 16, multi-dimensional shapes with unit dimensions -- in
double and single precision, and stores inputs and outputs in
golden_f64.npz / golden_f32.npz.  The reference ships no tests or golden
vectors of its own, so these files are the pinned record of its behaviour.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from minfft_b200._abi import OPS, shapes  # noqa: E402

SHAPES = [(1,), (2,), (4,), (8,), (16,), (32,), (64,), (256,), (1024,), (4, 8), (16, 32), (1, 8), (8, 1),
          (2, 4, 8), (8, 16, 4), (2, 1, 4), (2, 2, 4, 8)]


def key(op, dims, what):
    return f"{op}|{'x'.join(map(str, dims))}|{what}"


def make(single: bool, seed: int = 20240601):
    rng = np.random.default_rng(seed)
    out = {}
    rdt, cdt = oracle.np_dtypes(single)
    for dims in SHAPES:
        for op in OPS:
            ins, inc, _, _ = shapes(op, dims)
            x = rng.uniform(-1, 1, ins)
            if inc:
                x = x + 1j * rng.uniform(-1, 1, ins)
            x = x.astype(cdt if inc else rdt)
            y = oracle.apply(op, x, dims, single=single, kind="reference")
            out[key(op, dims, "in")] = x
            out[key(op, dims, "out")] = y
    return out


def main():
    if not oracle.available("reference"):
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` with the reference sources present")
    for single, name in ((False, "golden_f64.npz"), (True, "golden_f32.npz")):
        data = make(single)
        np.savez_compressed(os.path.join(HERE, name), **data)
        print(name, len(data) // 2, "cases")


if __name__ == "__main__":
    main()
