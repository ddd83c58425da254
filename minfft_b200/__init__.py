"""minfft_b200 -- a B200 (sm_100a) transform engine behind minfft's C API.

The product is the pair of shared libraries built from ``csrc/`` by
``python -m minfft_b200.build``:

* ``lib/libminfft_b200.so``        -- double precision (minfft's default)
* ``lib/libminfft_b200_single.so`` -- single precision (minfft's MINFFT_SINGLE)

Both export the 27 symbols of ``include/minfft.h`` (identical to the
reference minfft.h) plus the extensions of ``include/minfft_b200.h``.  This
module loads them with ctypes and offers thin conveniences for Python
callers (tests, the benchmark): every transform runs as CUDA kernels; there
is no CPU implementation here, and loading fails loudly when the library has
not been built.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

from ._abi import FAMILIES, OP_FAMILY, OPS, MinfftLibrary, shapes

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATHS = {False: os.path.join(LIB_DIR, "libminfft_b200.so"), True: os.path.join(LIB_DIR, "libminfft_b200_single.so")}
OP_CODES = {name: i for i, name in enumerate(OPS)}

PRECISIONS = {"fp32": 0, "tc_f16": 1, "tc_bf16": 2}  # minfft_b200.h MINFFT_B200_PREC_*
ERROR_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "EUNSUPPORTED", 5: "ETIMEOUT"}


class MinfftError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"minfft_b200 error {ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


class MixedJob(ctypes.Structure):
    """One job of a mixed batch (minfft_b200_job): transform code, length, device pointers."""

    _fields_ = [("op", ctypes.c_int), ("n", ctypes.c_int), ("inp", ctypes.c_void_p), ("out", ctypes.c_void_p)]


class Engine(MinfftLibrary):
    """One loaded engine library (one precision) with its extension API bound."""

    def __init__(self, single: bool = False):
        path = LIB_PATHS[bool(single)]
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m minfft_b200.build` "
                              "(the engine has no CPU fallback)")
        super().__init__(path, single)
        L = self.lib
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.minfft_b200_last_error.restype = i32
        L.minfft_b200_last_error.argtypes = []
        L.minfft_b200_last_error_message.restype = ctypes.c_char_p
        L.minfft_b200_last_error_message.argtypes = []
        L.minfft_b200_set_stream.argtypes = [vp, vp]
        L.minfft_b200_set_stream.restype = i32
        L.minfft_b200_get_stream.argtypes = [vp]
        L.minfft_b200_get_stream.restype = vp
        L.minfft_b200_synchronize.argtypes = [vp]
        L.minfft_b200_synchronize.restype = i32
        L.minfft_b200_execute_batch.argtypes = [i32, vp, vp, i32, vp]
        L.minfft_b200_execute_batch.restype = i32
        for f in ("minfft_b200_input_bytes", "minfft_b200_output_bytes", "minfft_b200_launch_count"):
            getattr(L, f).argtypes = [i32, vp]
            getattr(L, f).restype = i64 if f != "minfft_b200_launch_count" else i32
        L.minfft_b200_plan_bytes.argtypes = [vp]
        L.minfft_b200_plan_bytes.restype = i64
        L.minfft_b200_profile.argtypes = [vp, i32]
        L.minfft_b200_profile.restype = i32
        L.minfft_b200_profile_count.argtypes = [vp]
        L.minfft_b200_profile_count.restype = i32
        L.minfft_b200_profile_entry.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(i64),
                                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.minfft_b200_profile_entry.restype = i32
        L.minfft_b200_plan_selfcheck.argtypes = [i32, i32, ctypes.POINTER(i32), i32, i32, ctypes.c_char_p, i32,
                                                 ctypes.POINTER(i32)]
        L.minfft_b200_plan_selfcheck.restype = i32
        L.minfft_b200_plan_selfcheck_precision.argtypes = [i32, i32, ctypes.POINTER(i32), i32, i32, i32,
                                                           ctypes.c_char_p, i32, ctypes.POINTER(i32)]
        L.minfft_b200_plan_selfcheck_precision.restype = i32
        L.minfft_b200_set_precision.argtypes = [vp, i32]
        L.minfft_b200_set_precision.restype = i32
        L.minfft_b200_get_precision.argtypes = [vp]
        L.minfft_b200_get_precision.restype = i32
        L.minfft_b200_tc_status.argtypes = [vp]
        L.minfft_b200_tc_status.restype = i32
        L.minfft_b200_device_status.argtypes = [vp]
        L.minfft_b200_device_status.restype = i32
        L.minfft_b200_set_host_async.argtypes = [vp, i32]
        L.minfft_b200_set_host_async.restype = i32
        L.minfft_b200_autotune.argtypes = [vp, i32, i32, i32]
        L.minfft_b200_autotune.restype = i32
        for f in ("minfft_b200_tune_save", "minfft_b200_tune_load"):
            getattr(L, f).argtypes = [ctypes.c_char_p]
            getattr(L, f).restype = i32
        L.minfft_b200_tune_clear.argtypes = []
        L.minfft_b200_tune_clear.restype = i32
        L.minfft_b200_tune_size.argtypes = []
        L.minfft_b200_tune_size.restype = i32
        L.minfft_b200_tune_set_default.argtypes = [i32, i32, i32]
        L.minfft_b200_tune_set_default.restype = i32
        L.minfft_b200_mixed_plan.argtypes = [i32, ctypes.POINTER(MixedJob)]
        L.minfft_b200_mixed_plan.restype = vp
        L.minfft_b200_mixed_execute.argtypes = [vp, vp]
        L.minfft_b200_mixed_execute.restype = i32
        L.minfft_b200_mixed_autotune.argtypes = [vp, i32]
        L.minfft_b200_mixed_autotune.restype = i32
        L.minfft_b200_mixed_items.argtypes = [vp]
        L.minfft_b200_mixed_items.restype = i32
        L.minfft_b200_mixed_free.argtypes = [vp]
        L.minfft_b200_mixed_free.restype = None
        L.minfft_b200_test_fail_device_alloc.argtypes = [i64]
        L.minfft_b200_test_fail_device_alloc.restype = i32
        L.minfft_b200_test_device_alloc_count.argtypes = []
        L.minfft_b200_test_device_alloc_count.restype = i64
        L.minfft_b200_test_tc_withhold.argtypes = [i64]
        L.minfft_b200_test_tc_withhold.restype = i32

    # --------------------------------------------------------- errors
    def last_error(self) -> int:
        return int(self.lib.minfft_b200_last_error())

    def last_error_message(self) -> str:
        return self.lib.minfft_b200_last_error_message().decode()

    def check(self) -> None:
        """Raise MinfftError if the last call on this thread failed."""
        code = self.last_error()
        if code:
            raise MinfftError(code, self.last_error_message())

    # ------------------------------------------------------ extensions
    def set_stream(self, aux: int, stream: int) -> None:
        if self.lib.minfft_b200_set_stream(ctypes.c_void_p(aux), ctypes.c_void_p(stream or None)):
            self.check()

    def synchronize(self, aux: int) -> None:
        if self.lib.minfft_b200_synchronize(ctypes.c_void_p(aux)):
            self.check()

    def execute_batch(self, op: str, x: int, y: int, howmany: int, aux: int) -> None:
        rc = self.lib.minfft_b200_execute_batch(OP_CODES[op], ctypes.c_void_p(x), ctypes.c_void_p(y), howmany,
                                                ctypes.c_void_p(aux))
        if rc:
            self.check()

    def launch_count(self, op: str, aux: int) -> int:
        return int(self.lib.minfft_b200_launch_count(OP_CODES[op], ctypes.c_void_p(aux)))

    def plan_bytes(self, aux: int) -> int:
        return int(self.lib.minfft_b200_plan_bytes(ctypes.c_void_p(aux)))

    def plan_selfcheck(self, op: str, dims: Sequence[int], howmany: int = 1, alias: bool = False,
                       precision: str = "fp32"):
        """Host-only planning check (no device): (violations, report, launch count)."""
        arr = (ctypes.c_int * len(dims))(*[int(d) for d in dims])
        buf = ctypes.create_string_buffer(4096)
        n = ctypes.c_int(0)
        bad = self.lib.minfft_b200_plan_selfcheck_precision(OP_CODES[op], len(dims), arr, int(howmany), int(alias),
                                                            PRECISIONS[precision], buf, 4096, ctypes.byref(n))
        return int(bad), buf.value.decode(), int(n.value)

    def set_precision(self, aux: int, precision: str) -> None:
        """Arithmetic of the plan's complex 256-point passes: "fp32", "tc_f16" or "tc_bf16"."""
        if self.lib.minfft_b200_set_precision(ctypes.c_void_p(aux), PRECISIONS[precision]):
            self.check()

    def get_precision(self, aux: int) -> str:
        code = int(self.lib.minfft_b200_get_precision(ctypes.c_void_p(aux)))
        return {v: k for k, v in PRECISIONS.items()}[code]

    def set_host_async(self, aux: int, enable: bool = True) -> None:
        """Page-locked host arrays: calls return at once, ordered on the plan's stream."""
        if self.lib.minfft_b200_set_host_async(ctypes.c_void_p(aux), int(bool(enable))):
            self.check()

    def device_status(self, aux: int) -> None:
        """Raise if a kernel of the plan gave up on a bounded device-side wait since the last call."""
        if self.lib.minfft_b200_device_status(ctypes.c_void_p(aux)):
            self.check()

    def tc_status(self, aux: int) -> None:
        """Raise if a tensor-core pass of the plan gave up waiting since the last call."""
        if self.lib.minfft_b200_tc_status(ctypes.c_void_p(aux)):
            self.check()

    def autotune(self, aux: int, op: str, howmany: int = 1, reps: int = 5) -> None:
        """Tune every launch of `op` on this plan (kernel form, tile size) on the device."""
        if self.lib.minfft_b200_autotune(ctypes.c_void_p(aux), OP_CODES[op], int(howmany), int(reps)):
            self.check()

    def tune_save(self, path: str) -> None:
        if self.lib.minfft_b200_tune_save(path.encode()):
            self.check()

    def tune_load(self, path: str) -> None:
        if self.lib.minfft_b200_tune_load(path.encode()):
            self.check()

    def tune_clear(self) -> None:
        self.lib.minfft_b200_tune_clear()

    def tune_size(self) -> int:
        return int(self.lib.minfft_b200_tune_size())

    def tune_set_default(self, pipe: int = -1, cpb: int = 0, radix: int = 16) -> None:
        """Launch configuration where the tuning table has no entry (-1/0: planner's choice)."""
        self.lib.minfft_b200_tune_set_default(int(pipe), int(cpb), int(radix))

    def profile(self, aux: int, enable: int) -> None:
        if self.lib.minfft_b200_profile(ctypes.c_void_p(aux), int(enable)):
            self.check()

    def profile_stats(self, aux: int):
        """[(label, launches, total_ms, bytes_per_launch)] recorded since profiling was enabled."""
        n = self.lib.minfft_b200_profile_count(ctypes.c_void_p(aux))
        if n < 0:
            self.check()
        out = []
        for i in range(n):
            lab, cnt, ms, by = ctypes.c_char_p(), ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
            if self.lib.minfft_b200_profile_entry(ctypes.c_void_p(aux), i, ctypes.byref(lab), ctypes.byref(cnt),
                                                  ctypes.byref(ms), ctypes.byref(by)):
                self.check()
            out.append((lab.value.decode(), int(cnt.value), float(ms.value), float(by.value)))
        return out

    # ----------------------------------------------------- mixed batches
    def mixed_plan(self, jobs) -> int:
        """Plan a mixed batch from (op, n, in_ptr, out_ptr) tuples; returns the handle."""
        arr = (MixedJob * len(jobs))(*[MixedJob(OP_CODES[op] if isinstance(op, str) else int(op), int(n), int(i),
                                                int(o)) for op, n, i, o in jobs])
        h = self.lib.minfft_b200_mixed_plan(len(jobs), arr)
        if not h:
            code = self.last_error()
            raise MinfftError(code or 1, self.last_error_message())
        return int(h)

    def mixed_execute(self, handle: int, stream: int = 0) -> None:
        if self.lib.minfft_b200_mixed_execute(ctypes.c_void_p(handle), ctypes.c_void_p(stream or None)):
            self.check()

    def mixed_autotune(self, handle: int, reps: int = 3) -> None:
        if self.lib.minfft_b200_mixed_autotune(ctypes.c_void_p(handle), int(reps)):
            self.check()

    def mixed_items(self, handle: int) -> int:
        return int(self.lib.minfft_b200_mixed_items(ctypes.c_void_p(handle)))

    def mixed_free(self, handle: int) -> None:
        self.lib.minfft_b200_mixed_free(ctypes.c_void_p(handle))

    # ---------------------------------------------- checked plan API
    def plan(self, family: str, dims: Sequence[int]) -> "Plan":
        aux = self.mkaux(family, dims)
        if not aux:
            code = self.last_error()
            raise MinfftError(code or 1, self.last_error_message() or f"maker returned NULL for {tuple(dims)}")
        return Plan(self, family, tuple(int(d) for d in dims), aux)


class Plan:
    """An owned aux handle; ``plan(op, x, y)`` runs a transform on raw addresses."""

    def __init__(self, engine: Engine, family: str, dims, aux: int):
        self.engine, self.family, self.dims, self.aux = engine, family, dims, aux

    def __call__(self, op: str, x: int, y: int, check: bool = True) -> None:
        if OP_FAMILY[op] != self.family:
            raise ValueError(f"{op} needs a {OP_FAMILY[op]} plan, this is a {self.family} plan")
        self.engine.run(op, x, y, self.aux)
        if check:
            self.engine.check()

    def batch(self, op: str, x: int, y: int, howmany: int) -> None:
        self.engine.execute_batch(op, x, y, howmany, self.aux)

    def set_stream(self, stream: int) -> None:
        self.engine.set_stream(self.aux, stream)

    def set_host_async(self, enable: bool = True) -> None:
        self.engine.set_host_async(self.aux, enable)

    def synchronize(self) -> None:
        self.engine.synchronize(self.aux)

    def free(self) -> None:
        if self.aux:
            self.engine.free(self.aux)
            self.aux = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


_engines = {}


def engine(single: bool = False) -> Engine:
    """The process-wide engine of the given precision (loaded on first use)."""
    key = bool(single)
    if key not in _engines:
        _engines[key] = Engine(key)
    return _engines[key]


def torch_dtypes(single: bool):
    import torch

    return (torch.float32, torch.complex64) if single else (torch.float64, torch.complex128)


def transform(op: str, x, dims: Optional[Sequence[int]] = None, single: Optional[bool] = None, out=None):
    """Run ``op`` on a CUDA torch tensor through the C ABI and return the output tensor.

    ``dims`` defaults to ``x.shape`` (to the real shape for invrealdft it must
    be given).  The call is stream-ordered on the legacy default stream.
    """
    import torch

    if single is None:
        single = x.dtype in (torch.float32, torch.complex64)
    if dims is None:
        if op == "invrealdft":
            raise ValueError("invrealdft needs the real dims")
        dims = tuple(x.shape)
    in_shape, in_c, out_shape, out_c = shapes(op, dims)
    rdt, cdt = torch_dtypes(single)
    x = x.to(dtype=cdt if in_c else rdt).contiguous().reshape(in_shape)
    if out is None:
        out = torch.empty(out_shape, dtype=cdt if out_c else rdt, device=x.device)
    eng = engine(single)
    p = eng.plan(OP_FAMILY[op], dims)
    try:
        p(op, x.data_ptr(), out.data_ptr())
    finally:
        p.free()
    return out


__all__ = ["PRECISIONS", "ERROR_NAMES", "MixedJob", "Engine", "Plan", "MinfftError", "engine", "transform", "shapes", "OPS", "FAMILIES", "OP_FAMILY",
           "OP_CODES", "LIB_PATHS"]
