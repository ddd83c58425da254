"""The split column DFT of the 2-D DCT-2/DST-2 and DCT-3/DST-3 (dct_split.cu):
the radix-4 stage of the column DFT fused into an 8-row pass, Q-point column
DFTs on the block pairs {0, 2} and {1, 3}.  Against the double-precision
oracle, through the C ABI: every type-2/3 kind, several row counts and
lengths (Q = 128 .. 512 points per block), a batch of 2-D arrays in one call,
in place, host pointers.  Reference: minfft.c:692-887 (the 1-D kinds), :57-72 (the
multi-dimensional composition)."""
import numpy as np
import pytest

import minfft_b200
from conftest import rel_l2, tolerance
from test_gpu_parity import expected, gpu_apply, make_input

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def split_on(monkeypatch):
    """The split form is opt-in; plans made in these tests take it."""
    monkeypatch.setenv("MINFFT_B200_SPLITDCT", "1")

KINDS = ("dct2", "dst2", "dct3", "dst3")
SHAPES = [(1024, 128), (2048, 2048), (4096, 256), (1024, 2048)]


def plan_labels(eng, op, dims):
    plan = eng.plan(minfft_b200.OP_FAMILY[op], dims)
    try:
        n = int(np.prod(dims))
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        eng.profile(plan.aux, 1)
        plan(op, x.data_ptr(), y.data_ptr())
        return [s[0] for s in eng.profile_stats(plan.aux)]
    finally:
        plan.free()


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_split_dct_matches_oracle(single):
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(71)
    for dims in SHAPES:
        labs = plan_labels(eng, "dct2", dims)
        assert any(lab.startswith("dct_split<") for lab in labs), labs
        for op in KINDS:
            x = make_input(op, dims, rng, single, dist="normal")
            err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
            assert err <= tolerance(single, dims), (op, dims, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_split_dct_in_place_and_host(single):
    rng = np.random.default_rng(72)
    dims = (1024, 256)
    for op in KINDS:
        x = make_input(op, dims, rng, single)
        want = expected(op, x, dims)
        assert rel_l2(gpu_apply(op, x, dims, single, inplace=True), want) <= tolerance(single, dims), op
        assert rel_l2(gpu_apply(op, x, dims, single, host=True), want) <= tolerance(single, dims), op


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_split_dct_batch(single):
    """Three 1024 x 512 arrays in one call (minfft_b200_execute_batch)."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(73)
    dims, howmany = (1024, 512), 3
    rdt = torch.float32 if single else torch.float64
    for op in KINDS:
        xs = [make_input(op, dims, rng, single) for _ in range(howmany)]
        xt = torch.from_numpy(np.stack(xs)).cuda()
        yt = torch.full_like(xt, float("nan"))
        plan = eng.plan(minfft_b200.OP_FAMILY[op], dims)
        try:
            plan.batch(op, xt.data_ptr(), yt.data_ptr(), howmany)
            torch.cuda.synchronize()
        finally:
            plan.free()
        got = yt.cpu().numpy()
        for b in range(howmany):
            assert rel_l2(got[b], expected(op, xs[b], dims)) <= tolerance(single, dims), (op, b)
