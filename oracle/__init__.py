"""CPU oracle for the minfft transform family -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It is the checker, never the thing
measured or shipped: the product (``minfft_b200``) does not import it and has
no CPU path.

Two CPU implementations of the reference algorithms are available:

* ``restatement`` -- ``liboracle[_single].so`` built from ``minfft_oracle.c``,
  a plain-C restatement of reference minfft.c (always built by ``make``);
* ``reference`` -- ``_ref/libminfft_ref[_single].so``, the reference's own
  minfft.c compiled in place by ``oracle/Makefile`` (present where the
  reference sources were available at build time; the built files travel with
  the repository snapshot).

``apply(op, x, dims)`` runs one transform on numpy data and returns a new
array, so tests can write ``oracle.apply("dct2", x, (64, 32))``.
"""
from __future__ import annotations

import os
import subprocess
from typing import Optional, Sequence

import numpy as np

from minfft_b200._abi import OP_FAMILY, MinfftLibrary, shapes

HERE = os.path.dirname(os.path.abspath(__file__))
_PATHS = {
    ("restatement", False): os.path.join(HERE, "liboracle.so"),
    ("restatement", True): os.path.join(HERE, "liboracle_single.so"),
    ("reference", False): os.path.join(HERE, "_ref", "libminfft_ref.so"),
    ("reference", True): os.path.join(HERE, "_ref", "libminfft_ref_single.so"),
}
CPUBENCH_PATH = os.path.join(HERE, "libcpubench.so")
_cache = {}


def build(quiet: bool = True) -> None:
    """Compile the restatement, the CPU bench driver and (if its sources exist) the reference."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def available(kind: str = "restatement", single: bool = False) -> bool:
    return os.path.exists(_PATHS[(kind, bool(single))])


def library(kind: str = "restatement", single: bool = False) -> MinfftLibrary:
    key = (kind, bool(single))
    if key not in _cache:
        path = _PATHS[key]
        if not os.path.exists(path):
            if kind == "restatement":
                build()
            else:
                raise FileNotFoundError(f"{path} not built (reference sources were not available)")
        _cache[key] = MinfftLibrary(path, single)
    return _cache[key]


def best_kind() -> str:
    """The compiled reference where it was built, else the restatement."""
    return "reference" if available("reference") and available("reference", True) else "restatement"


def np_dtypes(single: bool):
    return (np.float32, np.complex64) if single else (np.float64, np.complex128)


def apply(op: str, x: np.ndarray, dims: Sequence[int], single: bool = False, kind: Optional[str] = None) -> np.ndarray:
    """Run reference-algorithm transform ``op`` on a copy of ``x`` (C order) and return the output."""
    kind = kind or "restatement"
    lib = library(kind, single)
    in_shape, in_cplx, out_shape, out_cplx = shapes(op, dims)
    rdt, cdt = np_dtypes(single)
    xin = np.ascontiguousarray(x, dtype=cdt if in_cplx else rdt).reshape(in_shape).copy()
    y = np.zeros(out_shape, dtype=cdt if out_cplx else rdt)
    aux = lib.mkaux(OP_FAMILY[op], dims)
    if not aux:
        raise ValueError(f"plan maker returned NULL for {op} {tuple(dims)}")
    try:
        lib.run(op, xin.ctypes.data, y.ctypes.data, aux)
    finally:
        lib.free(aux)
    return y


def apply_rows(op: str, rows, n: int, single: bool = False, kind: Optional[str] = None):
    """Run 1-D transform ``op`` of length ``n`` on every array in ``rows``
    with one plan (the reference's plans serve any number of calls); returns
    the list of outputs."""
    kind = kind or "restatement"
    lib = library(kind, single)
    in_shape, in_cplx, out_shape, out_cplx = shapes(op, (n,))
    rdt, cdt = np_dtypes(single)
    aux = lib.mkaux(OP_FAMILY[op], (n,))
    if not aux:
        raise ValueError(f"plan maker returned NULL for {op} ({n},)")
    outs = []
    try:
        for x in rows:
            xin = np.ascontiguousarray(x, dtype=cdt if in_cplx else rdt).reshape(in_shape).copy()
            y = np.zeros(out_shape, dtype=cdt if out_cplx else rdt)
            lib.run(op, xin.ctypes.data, y.ctypes.data, aux)
            outs.append(y)
    finally:
        lib.free(aux)
    return outs
