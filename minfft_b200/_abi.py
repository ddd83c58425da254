"""ctypes binding for the minfft C ABI (the 27 symbols of minfft.h).

One binding serves every library that exports that ABI: the GPU engine
(``libminfft_b200.so`` / ``libminfft_b200_single.so``), and -- in tests only --
the CPU oracle and the compiled reference.  Pointers are passed as plain
integers, so a caller may hand in host addresses (numpy ``.ctypes.data``) or
device addresses (``torch.Tensor.data_ptr()``).

Transform/plan pairing follows reference minfft.h:35-61 and README.md:
dft/invdft use a DFT plan, realdft/invrealdft a real-DFT plan, the four
type-2/3 transforms a t2t3 plan, the two type-4 transforms a t4 plan.
"""
from __future__ import annotations

import ctypes
from typing import Sequence, Tuple

OPS = ("dft", "invdft", "realdft", "invrealdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4")
FAMILIES = ("dft", "realdft", "t2t3", "t4")
OP_FAMILY = {
    "dft": "dft",
    "invdft": "dft",
    "realdft": "realdft",
    "invrealdft": "realdft",
    "dct2": "t2t3",
    "dst2": "t2t3",
    "dct3": "t2t3",
    "dst3": "t2t3",
    "dct4": "t4",
    "dst4": "t4",
}

_vp = ctypes.c_void_p
_int = ctypes.c_int


def bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    """Declare argument and result types of the 27 minfft.h symbols on ``lib``."""
    for op in OPS:
        f = getattr(lib, "minfft_" + op)
        f.argtypes = [_vp, _vp, _vp]
        f.restype = None
    for fam in FAMILIES:
        base = "minfft_mkaux_" + fam
        getattr(lib, base + "_1d").argtypes = [_int]
        getattr(lib, base + "_2d").argtypes = [_int, _int]
        getattr(lib, base + "_3d").argtypes = [_int, _int, _int]
        getattr(lib, base).argtypes = [_int, ctypes.POINTER(_int)]
        for suffix in ("_1d", "_2d", "_3d", ""):
            getattr(lib, base + suffix).restype = _vp
    lib.minfft_free_aux.argtypes = [_vp]
    lib.minfft_free_aux.restype = None
    return lib


def shapes(op: str, dims: Sequence[int]) -> Tuple[Tuple[int, ...], bool, Tuple[int, ...], bool]:
    """(input shape, input is complex, output shape, output is complex) of ``op`` on ``dims``.

    The real DFT maps an N1 x ... x Nd real array to N1 x ... x (Nd/2+1)
    complex values (reference README.md "Real DFT"); its inverse maps back.
    """
    dims = tuple(int(n) for n in dims)
    half = dims[:-1] + (dims[-1] // 2 + 1,)
    if op in ("dft", "invdft"):
        return dims, True, dims, True
    if op == "realdft":
        return dims, False, half, True
    if op == "invrealdft":
        return half, True, dims, False
    if op in OPS:
        return dims, False, dims, False
    raise ValueError(f"unknown transform {op!r}")


class MinfftLibrary:
    """A loaded library exporting the minfft ABI, with a small plan API."""

    def __init__(self, path: str, single: bool):
        self.path = path
        self.single = bool(single)
        self.lib = bind(ctypes.CDLL(path))

    def mkaux(self, family: str, dims: Sequence[int]) -> int:
        """Make a plan; returns the aux address, or 0 where the maker returned NULL."""
        if family not in FAMILIES:
            raise ValueError(f"unknown plan family {family!r}")
        base = "minfft_mkaux_" + family
        dims = [int(n) for n in dims]
        if len(dims) == 1:
            p = getattr(self.lib, base + "_1d")(dims[0])
        elif len(dims) == 2:
            p = getattr(self.lib, base + "_2d")(*dims)
        elif len(dims) == 3:
            p = getattr(self.lib, base + "_3d")(*dims)
        else:
            arr = (_int * max(len(dims), 1))(*dims)
            p = getattr(self.lib, base)(len(dims), arr)
        return int(p or 0)

    def mkaux_generic(self, family: str, dims: Sequence[int]) -> int:
        """Make a plan through the any-dimensional maker ``minfft_mkaux_<family>(d, Ns)``."""
        arr = (_int * max(len(dims), 1))(*[int(n) for n in dims])
        return int(getattr(self.lib, "minfft_mkaux_" + family)(len(dims), arr) or 0)

    def run(self, op: str, x: int, y: int, aux: int) -> None:
        getattr(self.lib, "minfft_" + op)(_vp(x), _vp(y), _vp(aux))

    def free(self, aux: int) -> None:
        self.lib.minfft_free_aux(_vp(aux) if aux else None)
