"""Failure paths of the makers and of the tensor-core pass, made on the host.

Allocation failures.  The reference's makers free a half-built plan whose
pointers were never initialised when a malloc fails (minfft.c:1065-1075 with
the free of minfft.c:1338-1347, reached from make_aux, minfft.c:1035-1052).
Here a test hook makes the k-th device allocation fail, for every k a maker
reaches, for all sixteen makers: each must return NULL, report
MINFFT_B200_ENOMEM, and leave the device's free memory where it was.
Nothing faults the GPU: the injected allocation is never made.
"""
import numpy as np
import pytest

import minfft_b200

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MAKERS = [(fam, dims) for fam in ("dft", "realdft", "t2t3", "t4")
          for dims in ((256,), (64, 32), (16, 8, 32), (8, 4, 16, 8))]
ENOMEM = 2


def free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("fam,dims", MAKERS, ids=[f"{f}-{len(d)}d" for f, d in MAKERS])
def test_maker_fails_cleanly_at_every_device_allocation(single, fam, dims):
    eng = minfft_b200.engine(single)
    L = eng.lib
    torch.cuda.init()
    # one successful make/free first: its allocations are counted, and any
    # one-time runtime state is set up before free memory is read
    assert L.minfft_b200_test_fail_device_alloc(0) == 0
    aux = eng.mkaux(fam, dims)
    assert aux, eng.last_error_message()
    count = L.minfft_b200_test_device_alloc_count()
    eng.free(aux)
    assert count >= 2  # the status word and at least one table or buffer
    base = free_bytes()
    try:
        for k in range(1, count + 1):
            eng.last_error()
            assert L.minfft_b200_test_fail_device_alloc(k) == 0
            aux = eng.mkaux(fam, dims)
            assert aux == 0, f"maker survived failure of allocation {k} of {count}"
            assert eng.last_error() == ENOMEM, (k, eng.last_error_message())
            assert free_bytes() == base, f"allocation {k} of {count}: device memory leaked"
    finally:
        L.minfft_b200_test_fail_device_alloc(0)
    # the library still works afterwards
    aux = eng.mkaux(fam, dims)
    assert aux
    eng.free(aux)
    assert free_bytes() == base


def test_tc_wait_timeout_is_reported_and_the_plan_recovers():
    """The tensor-core pass waits for its matrix operations with a bounded
    poll.  A test hook withholds the first stage's operations (a completion
    nothing will signal) and shortens that wait; the launch must give up,
    record MINFFT_B200_ETIMEOUT for minfft_b200_device_status, free its
    tensor memory and leave the context usable: the same plan then gives
    correct results."""
    import oracle
    from conftest import rel_l2

    eng = minfft_b200.engine(True)
    L = eng.lib
    dims = (64, 256)
    rng = np.random.default_rng(12)
    x = (rng.uniform(-1, 1, dims) + 1j * rng.uniform(-1, 1, dims)).astype(np.complex64)
    xt = torch.from_numpy(x).cuda()
    y = torch.zeros_like(xt)
    plan = eng.plan("dft", dims)
    try:
        eng.set_precision(plan.aux, "tc_f16")
        assert L.minfft_b200_device_status(plan.aux) == 0
        assert L.minfft_b200_test_tc_withhold(256) == 0
        try:
            plan("dft", xt.data_ptr(), y.data_ptr())
            assert L.minfft_b200_device_status(plan.aux) == 5  # MINFFT_B200_ETIMEOUT
            assert eng.last_error() == 5  # also the thread's last error (read and cleared here)
        finally:
            L.minfft_b200_test_tc_withhold(0)
        assert L.minfft_b200_device_status(plan.aux) == 0  # the record was cleared
        plan("dft", xt.data_ptr(), y.data_ptr())
        assert L.minfft_b200_device_status(plan.aux) == 0
        ref = oracle.apply("dft", x.astype(np.complex128), dims, kind=oracle.best_kind())
        assert rel_l2(y.cpu().numpy(), ref) <= 1e-6
    finally:
        plan.free()
