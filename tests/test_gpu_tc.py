"""Tensor-core split-precision passes (minfft_b200_set_precision) against the
double-precision oracle, through the C ABI of the single-precision library.

Every complex 256-point axis runs on tcgen05 in the TC modes: rows and
columns of 1-D to 3-D arrays, ragged batches (ending inside a CTA tile),
in-place calls, inverse transforms, and the 256-point passes of Stockham
chains over HBM (the first, and the pre-twiddled later ones).  Bar: relative L2 error against the FP64 oracle at most 1e-6
(tighter than the FP32 bar of 1e-6 * log2 N), and no wait of the kernel ran
out (minfft_b200_tc_status)."""
import numpy as np
import pytest

import minfft_b200
import oracle
from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MODES = ("tc_f16", "tc_bf16")
TC_BAR = 1e-6


def run(op, x, dims, mode, inplace=False):
    eng = minfft_b200.engine(True)
    plan = eng.plan("dft", dims)
    try:
        eng.set_precision(plan.aux, mode)
        assert eng.get_precision(plan.aux) == mode
        xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        if inplace:
            plan(op, xt.data_ptr(), xt.data_ptr())
            y = xt
        else:
            y = torch.full(x.shape, float("nan"), dtype=torch.complex64, device="cuda")
            plan(op, xt.data_ptr(), y.data_ptr())
        eng.tc_status(plan.aux)
        torch.cuda.synchronize()
        return y.cpu().numpy()
    finally:
        plan.free()


def labels(dims, mode, op="dft"):
    """Kernel labels one call of the plan launches (via launch-level timing)."""
    eng = minfft_b200.engine(True)
    plan = eng.plan("dft", dims)
    try:
        eng.set_precision(plan.aux, mode)
        x = torch.zeros(dims, dtype=torch.complex64, device="cuda")
        eng.profile(plan.aux, 1)
        plan(op, x.data_ptr(), x.data_ptr())
        return [s[0] for s in eng.profile_stats(plan.aux)]
    finally:
        plan.free()


def data(dims, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(dims) + 1j * rng.standard_normal(dims)).astype(np.complex64)


def ref(op, x, dims):
    return oracle.apply(op, x.astype(np.complex128), dims, single=False, kind=oracle.best_kind())


SHAPES = [(256,), (2, 256), (32, 256), (256, 2), (256, 16), (256, 256), (2, 256, 256), (256, 4, 256),
          (64, 64, 256), (256, 16, 4)]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims", SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_tc_dft_matches_oracle(mode, dims):
    x = data(dims, 1)
    for op in ("dft", "invdft"):
        got = run(op, x, dims, mode)
        err = rel_l2(got, ref(op, x, dims))
        assert err <= TC_BAR, (op, mode, dims, err)


@pytest.mark.parametrize("mode", MODES)
def test_tc_in_place(mode):
    dims = (32, 256)
    x = data(dims, 2)
    got = run("dft", x.copy(), dims, mode, inplace=True)
    assert rel_l2(got, ref("dft", x, dims)) <= TC_BAR


@pytest.mark.parametrize("mode", MODES)
def test_tc_uses_tensor_core_kernels(mode):
    names = labels((64, 256), mode)
    assert any(n.startswith(("tc_pass<", "tc_stream<")) for n in names), names
    assert not any(n.startswith("axis_pass<cplx,L=256") for n in names), names
    # back to FP32: no tensor-core launch
    eng = minfft_b200.engine(True)
    plan = eng.plan("dft", (64, 256))
    try:
        eng.set_precision(plan.aux, mode)
        eng.set_precision(plan.aux, "fp32")
        x = torch.zeros((64, 256), dtype=torch.complex64, device="cuda")
        eng.profile(plan.aux, 1)
        plan("dft", x.data_ptr(), x.data_ptr())
        assert not any(s[0].startswith(("tc_pass<", "tc_stream<")) for s in eng.profile_stats(plan.aux))
    finally:
        plan.free()


@pytest.mark.parametrize("mode", MODES)
def test_tc_passes_of_long_column_axis(mode):
    """65536-point columns: two HBM passes of 256, both on tensor cores."""
    dims = (65536, 2)
    names = labels(dims, mode)
    assert any(n.startswith(("tc_pass<", "tc_stream<")) for n in names), names
    x = data(dims, 3)
    got = run("dft", x, dims, mode)
    err = rel_l2(got, ref("dft", x, dims))
    assert err <= 2 * TC_BAR, err


# (dims, tensor-core launches per call): 2^16 = 256 x 256 (both passes, the
# second pre-twiddled), 2^20 = 256 x 4096, 2^25 = 256 x 256 x 512, and
# 131072-point columns of four = 256 x 512
LONG_CHAINS = [((1 << 16,), 2), ((1 << 20,), 1), ((1 << 25,), 2), ((1 << 17, 4), 1)]


def tc_launches(dims, mode, op="dft"):
    eng = minfft_b200.engine(True)
    plan = eng.plan("dft", dims)
    try:
        eng.set_precision(plan.aux, mode)
        x = torch.zeros(dims, dtype=torch.complex64, device="cuda")
        y = torch.empty_like(x)
        eng.profile(plan.aux, 1)
        plan(op, x.data_ptr(), y.data_ptr())
        return sum(s[1] for s in eng.profile_stats(plan.aux) if s[0].startswith(("tc_pass<", "tc_stream<")))
    finally:
        plan.free()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dims,ntc", LONG_CHAINS, ids=["x".join(map(str, d)) for d, _ in LONG_CHAINS])
def test_tc_passes_of_long_chains(dims, ntc, mode):
    """Axes beyond one CTA run as Stockham chains over HBM; in a TC mode the
    chain holds as many 256-point passes as its pass count allows, all on
    tensor cores, the later ones pre-twiddled in FP32 before the split."""
    assert tc_launches(dims, mode) == ntc
    x = data(dims, 11)
    for op in ("dft", "invdft"):
        got = run(op, x, dims, mode)
        err = rel_l2(got, ref(op, x, dims))
        assert err <= 2 * TC_BAR, (op, err)


def run_rows(op, x, mode):
    """A batch of 256-point transforms (rows of x) through one 1-D plan."""
    eng = minfft_b200.engine(True)
    plan = eng.plan("dft", (256,))
    try:
        eng.set_precision(plan.aux, mode)
        xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        y = torch.empty_like(xt)
        plan.batch(op, xt.data_ptr(), y.data_ptr(), x.shape[0])
        eng.tc_status(plan.aux)
        return y.cpu().numpy()
    finally:
        plan.free()


# (points, post-rotation as a separate element-wise step): the half-length
# chains 256 x 128 and 256 x 512 end in a CUDA-core pass that takes the
# post-rotation into its store; 256 x 256 ends on the tensor cores and
# 256 x 2048 in a pass longer than 1024 points, so both keep the step.
T4_CHAINS = [(1 << 16, False), (1 << 17, True), (1 << 18, False), (1 << 20, True)]


def run_t4(op, x, mode):
    """One DCT-4 / DST-4 line of x in a TC mode; also the kernel labels of
    one call (launch-level timing, on a zero input)."""
    eng = minfft_b200.engine(True)
    n = x.size
    plan = eng.plan("t4", (n,))
    try:
        eng.set_precision(plan.aux, mode)
        z = torch.zeros(n, dtype=torch.float32, device="cuda")
        zo = torch.zeros_like(z)
        eng.profile(plan.aux, 1)
        plan(op, z.data_ptr(), zo.data_ptr())
        labs = [s[0] for s in eng.profile_stats(plan.aux)]
        eng.profile(plan.aux, 0)
        xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        y = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
        plan(op, xt.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        eng.tc_status(plan.aux)
        return y.cpu().numpy(), labs
    finally:
        plan.free()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n,line_post", T4_CHAINS, ids=[f"2^{n.bit_length() - 1}" for n, _ in T4_CHAINS])
def test_tc_type4_chains(n, line_post, mode):
    """DCT-4 / DST-4 lines whose half-length DFT is a Stockham chain with
    tensor-core passes: the pre-rotation as an element-wise step (paired
    points n, L-1-n), the post-rotation fused into a last CUDA-core pass of
    128 to 1024 points, or else an element-wise step after the chain."""
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    for op in ("dct4", "dst4"):
        got, labs = run_t4(op, x, mode)
        assert any(("tc_stream<" in lab or "tc_pass<" in lab) for lab in labs), labs
        assert any("line<t4_pre>" in lab for lab in labs), labs
        assert any("line<t4_post>" in lab for lab in labs) == line_post, labs
        want = oracle.apply(op, x.astype(np.float64), (n,), single=False, kind=oracle.best_kind())
        err = rel_l2(got, want)
        assert err <= TC_BAR, (op, n, mode, err)


@pytest.mark.parametrize("mode", MODES)
def test_tc_wide_dynamic_range(mode):
    """Per-row block scaling keeps every transform of a batch accurate when
    their magnitudes differ by many orders (64 x 256-point batch)."""
    rng = np.random.default_rng(4)
    x = (data((64, 256), 4) * np.exp(rng.uniform(-20, 20, (64, 1)))).astype(np.complex64)
    got = run_rows("dft", x, mode)
    for i in range(x.shape[0]):
        assert rel_l2(got[i], ref("dft", x[i], (256,))) <= TC_BAR, i


@pytest.mark.parametrize("mode", MODES)
def test_tc_ragged_batches(mode):
    """Batches that end inside a CTA tile: 37 rows; 3 arrays of 256 x 2
    (6 columns of 256 points)."""
    x = data((37, 256), 6)
    for op in ("dft", "invdft"):
        got = run_rows(op, x, mode)
        for i in range(x.shape[0]):
            assert rel_l2(got[i], ref(op, x[i], (256,))) <= TC_BAR, (op, i)
    eng = minfft_b200.engine(True)
    plan = eng.plan("dft", (256, 2))
    x = data((3, 256, 2), 7)
    try:
        eng.set_precision(plan.aux, mode)
        xt = torch.from_numpy(x).cuda()
        y = torch.empty_like(xt)
        plan.batch("dft", xt.data_ptr(), y.data_ptr(), 3)
        eng.tc_status(plan.aux)
        got = y.cpu().numpy()
    finally:
        plan.free()
    for i in range(3):
        assert rel_l2(got[i], ref("dft", x[i], (256, 2))) <= TC_BAR, i


@pytest.mark.parametrize("mode", MODES)
def test_tc_zero_rows_and_exact_tones(mode):
    x = np.zeros((16, 256), np.complex64)
    x[3, 7] = 1.0
    x[5] = np.exp(2j * np.pi * 9 * np.arange(256) / 256).astype(np.complex64)
    got = run_rows("dft", x, mode)
    assert np.all(got[0] == 0) and np.all(got[15] == 0)
    for i in (3, 5):
        assert np.max(np.abs(got[i] - ref("dft", x[i], (256,)))) < 1e-4, (mode, i)


def test_tc_double_library_rejects_tensor_core_modes():
    eng = minfft_b200.engine(False)
    plan = eng.plan("dft", (256,))
    try:
        with pytest.raises(minfft_b200.MinfftError) as e:
            eng.set_precision(plan.aux, "tc_f16")
        assert e.value.code == 4
        assert eng.get_precision(plan.aux) == "fp32"
    finally:
        plan.free()
