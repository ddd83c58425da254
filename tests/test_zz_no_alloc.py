"""The allocation-free DFT entry point (minfft_b200_dft_noalloc).

It exists for callers that cannot allocate device memory -- their GPU memory
is owned by another allocator's pool or a fixed budget, or an allocation's
latency and implied synchronisation are unacceptable in their loop -- and so
cannot hold a plan.  These tests call it through the C ABI and check that it
agrees with the planned entry point (minfft_mkaux_dft_1d + minfft_dft /
minfft_invdft) and with the double-precision oracle within the parity
tolerance, on two calls in a row (the calls share the static scratch array,
so the second must not see stale state), that a call takes no device memory,
and that lengths beyond its fixed maximum, host memory and another device's
memory are refused with an error.

This file sorts last so that a run stopping at the first failure has run
every other test first; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import minfft_b200
import oracle
from conftest import rel_l2, tolerance

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MAX_N = 1 << 18


def noalloc_fn(eng):
    f = eng.lib.minfft_b200_dft_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def planned(eng, x, inverse):
    n = x.numel()
    y = torch.empty_like(x)
    p = eng.plan("dft", (n,))
    p("invdft" if inverse else "dft", x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    p.free()
    return y


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_noalloc_matches_planned_dft_on_consecutive_calls(single):
    eng = minfft_b200.engine(single)
    f = noalloc_fn(eng)
    cdt = torch.complex64 if single else torch.complex128
    rng = np.random.default_rng(99)
    # two calls in a row with different lengths and directions, then a
    # third repeating the first length: the shared scratch carries no state
    for n, inverse in ((MAX_N, 0), (1 << 13, 1), (MAX_N, 1), (4, 0)):
        x = torch.from_numpy(rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).to("cuda", cdt)
        y = torch.full_like(x, complex("nan+nanj"))
        rc = f(x.data_ptr(), y.data_ptr(), n, inverse, None)
        assert rc == 0, eng.last_error_message()
        torch.cuda.synchronize()
        ref = planned(eng, x, inverse)
        err = rel_l2(y.cpu().numpy(), ref.cpu().numpy())
        assert err <= tolerance(single, (n,)), (n, inverse, err)
        # and against the oracle on the same (upcast) input
        want = oracle.apply("invdft" if inverse else "dft", x.cpu().numpy().astype(np.complex128), (n,),
                            kind=oracle.best_kind())
        err = rel_l2(y.cpu().numpy(), want)
        assert err <= tolerance(single, (n,)), (n, inverse, err)


def test_noalloc_takes_no_device_memory():
    eng = minfft_b200.engine(False)
    f = noalloc_fn(eng)
    x = torch.randn(MAX_N, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    assert f(x.data_ptr(), y.data_ptr(), MAX_N, 0, None) == 0  # first call: set-up on this device
    torch.cuda.synchronize()
    before_torch = torch.cuda.memory_allocated()
    before_free = torch.cuda.mem_get_info()[0]
    for inverse in (0, 1):
        assert f(x.data_ptr(), y.data_ptr(), MAX_N, inverse, None) == 0, eng.last_error_message()
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == before_torch
    assert torch.cuda.mem_get_info()[0] == before_free


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2, reason="needs two devices")
def test_noalloc_refuses_another_devices_memory():
    eng = minfft_b200.engine(False)
    f = noalloc_fn(eng)
    torch.cuda.set_device(0)
    other = torch.zeros(64, dtype=torch.complex128, device="cuda:1")
    assert f(other.data_ptr(), other.data_ptr(), 64, 0, None) == 1  # MINFFT_B200_EINVAL, nothing launched
    assert "current device" in eng.last_error_message()


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_noalloc_in_place(single):
    eng = minfft_b200.engine(single)
    f = noalloc_fn(eng)
    cdt = torch.complex64 if single else torch.complex128
    n = 1 << 16
    x = torch.randn(n, dtype=cdt, device="cuda")
    ref = planned(eng, x, 0)
    buf = x.clone()
    assert f(buf.data_ptr(), buf.data_ptr(), n, 0, None) == 0
    torch.cuda.synchronize()
    assert rel_l2(buf.cpu().numpy(), ref.cpu().numpy()) <= tolerance(single, (n,))


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_noalloc_refuses_lengths_beyond_its_maximum(single):
    eng = minfft_b200.engine(single)
    f = noalloc_fn(eng)
    x = torch.zeros(2 * MAX_N, dtype=torch.complex128, device="cuda")
    eng.last_error()
    for bad in (2 * MAX_N, 3 * 1024, 2, 0, -8):
        assert f(x.data_ptr(), x.data_ptr(), bad, 0, None) == 1  # MINFFT_B200_EINVAL
        assert eng.last_error() == 1
        assert "262144" in eng.last_error_message() or bad <= 2
    host = np.zeros(64, dtype=np.complex128)
    assert f(host.ctypes.data, host.ctypes.data, 32, 0, None) == 1  # host memory is refused, not touched
