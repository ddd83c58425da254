"""GPU engine parity against the CPU oracle, through the C ABI.

Every transform, 1-D to 4-D, both precisions, edge sizes (the reference's
N = 1, 2, 4, 8 codelets, N = 16, unit dimensions), the multi-pass lengths
beyond one CTA, in-place calls, host-pointer staging, batching, and error
reporting.  Bars (relative L2 against the double-precision oracle on the same
inputs): 1e-13 for the double library, 1e-6 * log2(N) for the single one.
"""
import ctypes

import numpy as np
import pytest

import minfft_b200
import oracle
from conftest import rel_l2, tolerance
from minfft_b200 import OP_FAMILY, OPS, shapes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def oracle_kind():
    return oracle.best_kind()


def make_input(op, dims, rng, single, dist="uniform"):
    ins, inc, _, _ = shapes(op, dims)
    draw = (lambda s: rng.uniform(-1, 1, s)) if dist == "uniform" else (lambda s: rng.standard_normal(s))
    x = draw(ins)
    if inc:
        x = x + 1j * draw(ins)
    rdt, cdt = oracle.np_dtypes(single)
    return x.astype(cdt if inc else rdt)


def expected(op, x, dims):
    """Double-precision oracle result for input x (upcast)."""
    x64 = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    return oracle.apply(op, x64, dims, single=False, kind=oracle_kind())


def gpu_apply(op, x, dims, single, inplace=False, host=False):
    eng = minfft_b200.engine(single)
    _, _, out_shape, out_c = shapes(op, dims)
    rdt, cdt = oracle.np_dtypes(single)
    plan = eng.plan(OP_FAMILY[op], dims)
    try:
        if host:
            xh = np.ascontiguousarray(x).copy()
            if inplace:
                nbytes = max(xh.nbytes, int(np.prod(out_shape)) * np.dtype(cdt if out_c else rdt).itemsize)
                buf = np.zeros(nbytes // 8 + 2, dtype=np.float64)
                raw = buf.view(np.uint8)[: xh.nbytes]
                raw[:] = xh.view(np.uint8).ravel()
                plan(op, buf.ctypes.data, buf.ctypes.data)
                return buf.view(np.uint8)[: int(np.prod(out_shape)) * np.dtype(cdt if out_c else rdt).itemsize].view(
                    cdt if out_c else rdt).reshape(out_shape)
            y = np.zeros(out_shape, dtype=cdt if out_c else rdt)
            plan(op, xh.ctypes.data, y.ctypes.data)
            return y
        xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        if inplace:
            nbytes = max(xt.numel() * xt.element_size(),
                         int(np.prod(out_shape)) * np.dtype(cdt if out_c else rdt).itemsize)
            buf = torch.zeros(nbytes // 8 + 2, dtype=torch.float64, device="cuda")
            buf.view(torch.uint8)[: xt.numel() * xt.element_size()].copy_(xt.view(torch.uint8).flatten())
            plan(op, buf.data_ptr(), buf.data_ptr())
            torch.cuda.synchronize()
            nb = int(np.prod(out_shape)) * np.dtype(cdt if out_c else rdt).itemsize
            return buf.view(torch.uint8)[:nb].cpu().numpy().view(cdt if out_c else rdt).reshape(out_shape)
        tdt = {np.float32: torch.float32, np.float64: torch.float64, np.complex64: torch.complex64,
               np.complex128: torch.complex128}[cdt if out_c else rdt]
        y = torch.full(out_shape, float("nan"), dtype=tdt, device="cuda")  # unwritten outputs stay NaN
        plan(op, xt.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(xt.cpu(), torch.from_numpy(np.ascontiguousarray(x))), "input was modified"
        return y.cpu().numpy()
    finally:
        plan.free()


SMALL_SHAPES = [(1,), (2,), (4,), (8,), (16,), (32,), (64,), (128,), (256,), (512,), (1024,), (4096,), (4, 8),
                (16, 32), (1, 8), (8, 1), (64, 128), (2, 4, 8), (8, 16, 4), (2, 1, 4), (1, 2, 1), (2, 2, 4, 8),
                (32, 32, 32)]


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("dims", SMALL_SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_parity_small(dims, single):
    rng = np.random.default_rng(hash(dims) % (2**32))
    for op in OPS:
        x = make_input(op, dims, rng, single)
        got = gpu_apply(op, x, dims, single)
        ref = expected(op, x, dims)
        err = rel_l2(got, ref)
        assert err <= tolerance(single, dims), (op, dims, err)


def test_parity_against_golden_vectors():
    """The engine reproduces the reference's own outputs (tests/golden)."""
    import os

    for single, name in ((False, "golden_f64.npz"), (True, "golden_f32.npz")):
        data = np.load(os.path.join(os.path.dirname(__file__), "golden", name))
        for k in data.files:
            op, d, what = k.split("|")
            if what != "in":
                continue
            dims = tuple(int(v) for v in d.split("x"))
            got = gpu_apply(op, data[k], dims, single)
            ref = data[f"{op}|{d}|out"]
            # golden outputs are the reference's own precision: compare at that precision
            tol = 5e-7 * max(1, np.log2(max(np.prod(dims), 2))) if single else 1e-13
            assert rel_l2(got, ref) <= tol, (op, dims, single)


LONG_1D = [8192, 16384, 32768, 65536, 1 << 20]


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("n", LONG_1D)
def test_parity_long_1d(n, single):
    """Lengths beyond one CTA: the HBM Stockham passes and the standalone
    pre/post kernels of the real transforms."""
    rng = np.random.default_rng(n)
    dims = (n,)
    for op in OPS:
        x = make_input(op, dims, rng, single)
        err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
        assert err <= tolerance(single, dims), (op, n, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("n", [1 << 21, 1 << 22])
def test_parity_three_pass_chains(n, single):
    """The CUDA-core chains cap their passes over HBM at 1024 points, so
    2^21 .. 2^24-point axes take three passes (for the real kinds, of their
    half-length complex DFT): every transform kind against the oracle."""
    rng = np.random.default_rng(n + 3)
    dims = (n,)
    for op in OPS:
        x = make_input(op, dims, rng, single)
        err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
        assert err <= tolerance(single, dims), (op, n, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("dims", [(8192, 4), (4, 8192), (2, 16384), (16384, 2), (8, 8, 8192)],
                         ids=lambda d: "x".join(map(str, d)))
def test_parity_long_axes_multid(dims, single):
    rng = np.random.default_rng(5)
    for op in OPS:
        x = make_input(op, dims, rng, single)
        err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
        assert err <= tolerance(single, dims), (op, dims, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("dims", [(16,), (1024,), (32768,), (16, 32), (8, 4, 16), (4096, 8)],
                         ids=lambda d: "x".join(map(str, d)))
def test_in_place_equals_out_of_place(dims, single):
    """README "Interface": routines work in place; the real DFT buffer must
    hold the (larger) output."""
    rng = np.random.default_rng(17)
    for op in OPS:
        x = make_input(op, dims, rng, single)
        a = gpu_apply(op, x, dims, single)
        b = gpu_apply(op, x, dims, single, inplace=True)
        assert rel_l2(b, a) <= (1e-15 if not single else 1e-7), (op, dims)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("dims", [(8,), (4096,), (65536,), (16, 32)], ids=lambda d: "x".join(map(str, d)))
def test_host_pointers_are_staged(dims, single):
    """Unmodified reference callers pass host arrays; the engine stages them."""
    rng = np.random.default_rng(23)
    for op in OPS:
        x = make_input(op, dims, rng, single)
        got = gpu_apply(op, x, dims, single, host=True)
        assert rel_l2(got, expected(op, x, dims)) <= tolerance(single, dims), (op, dims)
        got = gpu_apply(op, x, dims, single, host=True, inplace=True)
        assert rel_l2(got, expected(op, x, dims)) <= tolerance(single, dims), (op, dims, "in place")


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_batch_api_matches_single_calls(single):
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(29)
    howmany = 5
    for dims in [(64,), (16, 8)]:
        for op in OPS:
            ins, inc, outs, outc = shapes(op, dims)
            xs = np.stack([make_input(op, dims, rng, single) for _ in range(howmany)])
            rdt, cdt = oracle.np_dtypes(single)
            xt = torch.from_numpy(xs).cuda()
            tdt = torch.complex64 if single else torch.complex128
            if not outc:
                tdt = torch.float32 if single else torch.float64
            yt = torch.empty((howmany,) + outs, dtype=tdt, device="cuda")
            plan = eng.plan(OP_FAMILY[op], dims)
            plan.batch(op, xt.data_ptr(), yt.data_ptr(), howmany)
            torch.cuda.synchronize()
            plan.free()
            for i in range(howmany):
                assert rel_l2(yt[i].cpu().numpy(), expected(op, xs[i], dims)) <= tolerance(single, dims)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_wrong_plan_kind_is_rejected(single):
    eng = minfft_b200.engine(single)
    p = eng.plan("t4", (16,))
    x = torch.zeros(32, dtype=torch.float64, device="cuda")
    eng.last_error()
    eng.run("dft", x.data_ptr(), x.data_ptr(), p.aux)
    assert eng.last_error() == 1
    eng.run("dct2", x.data_ptr(), x.data_ptr(), p.aux)
    assert eng.last_error() == 1
    eng.run("dct4", x.data_ptr(), x.data_ptr(), p.aux)
    assert eng.last_error() == 0
    p.free()


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_misaligned_complex_data_is_rejected(single):
    eng = minfft_b200.engine(single)
    p = eng.plan("dft", (64,))
    x = torch.zeros(300, dtype=torch.float64, device="cuda")
    eng.last_error()
    eng.run("dft", x.data_ptr() + 4, x.data_ptr() + 4, p.aux)  # not a multiple of 8/16 bytes
    assert eng.last_error() == 1
    p.free()


def test_round_trips_scale_as_documented():
    rng = np.random.default_rng(31)
    dims = (64, 32)
    n = 64 * 32
    xc = make_input("dft", dims, rng, False)
    xr = make_input("dct2", dims, rng, False)
    y = gpu_apply("invdft", gpu_apply("dft", xc, dims, False), dims, False)
    assert rel_l2(y / n, xc) < 1e-14
    y = gpu_apply("invrealdft", gpu_apply("realdft", xr, dims, False), dims, False)
    assert rel_l2(y / n, xr) < 1e-14
    y = gpu_apply("dct3", gpu_apply("dct2", xr, dims, False), dims, False)
    assert rel_l2(y / (4 * n), xr) < 1e-14
    y = gpu_apply("dst4", gpu_apply("dst4", xr, dims, False), dims, False)
    assert rel_l2(y / (4 * n), xr) < 1e-14


SPLIT_2D = [(1024, 32), (1024, 64), (2048, 256), (4096, 32), (1024, 4096)]


def launch_labels(eng, plan, op, x_dev, y_dev):
    eng.profile(plan.aux, 1)
    plan(op, x_dev.data_ptr(), y_dev.data_ptr())
    torch.cuda.synchronize()
    labels = [st[0] for st in eng.profile_stats(plan.aux)]
    eng.profile(plan.aux, 0)
    return labels


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("dims", SPLIT_2D, ids=lambda d: "x".join(map(str, d)))
def test_split_column_real_dft_2d(dims, single):
    """2-D real DFTs of at least 1024 rows split their column DFT: a radix-4
    stage across rows j + Q*m fused into the row pass, length-rows/4 column
    passes.  The launch list shows both fused kernels, and forward, inverse,
    in-place, host-pointer and batched calls match the oracle, also after
    autotuning (which keeps four rows per CTA)."""
    rng = np.random.default_rng(sum(dims))
    tol = tolerance(single, dims)
    eng = minfft_b200.engine(single)
    x = make_input("realdft", dims, rng, single)
    z = make_input("invrealdft", dims, rng, single)
    plan = eng.plan("realdft", dims)
    try:
        xt = torch.from_numpy(x).cuda()
        zt = torch.from_numpy(z).cuda()
        yt = torch.empty(z.shape, dtype=zt.dtype, device="cuda")
        wt = torch.empty(x.shape, dtype=xt.dtype, device="cuda")
        assert any(lab.startswith("axis_pass<r2c+col4") for lab in launch_labels(eng, plan, "realdft", xt, yt))
        assert any(lab.startswith("axis_pass<col4+c2r") for lab in launch_labels(eng, plan, "invrealdft", zt, wt))
        for _ in range(2):  # as planned, then with the autotuner's configurations
            plan("realdft", xt.data_ptr(), yt.data_ptr())
            plan("invrealdft", zt.data_ptr(), wt.data_ptr())
            torch.cuda.synchronize()
            assert rel_l2(yt.cpu().numpy(), expected("realdft", x, dims)) <= tol
            assert rel_l2(wt.cpu().numpy(), expected("invrealdft", z, dims)) <= tol
            assert torch.equal(zt.cpu(), torch.from_numpy(z)), "inverse input was modified"
            eng.autotune(plan.aux, "realdft", 1, 2)
            eng.autotune(plan.aux, "invrealdft", 1, 2)
        # a batch of three arrays through one call
        xb = np.stack([make_input("realdft", dims, rng, single) for _ in range(3)])
        xbt = torch.from_numpy(xb).cuda()
        ybt = torch.empty((3,) + z.shape, dtype=zt.dtype, device="cuda")
        plan.batch("realdft", xbt.data_ptr(), ybt.data_ptr(), 3)
        torch.cuda.synchronize()
        yb = ybt.cpu().numpy()
        for i in range(3):
            assert rel_l2(yb[i], expected("realdft", xb[i], dims)) <= tol, i
    finally:
        plan.free()
    for op, inp in (("realdft", x), ("invrealdft", z)):
        ref = expected(op, inp, dims)
        assert rel_l2(gpu_apply(op, inp, dims, single, inplace=True), ref) <= tol, (op, "in place")
        assert rel_l2(gpu_apply(op, inp, dims, single, host=True), ref) <= tol, (op, "host")
    y = gpu_apply("invrealdft", gpu_apply("realdft", x.astype(np.float64), dims, False), dims, False)
    assert rel_l2(y / np.prod(dims), x) < 1e-14


# --------------------------------------------------------- workload sizes
@pytest.mark.slow
@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_config_2d_2048(single):
    """2048 x 2048 real DFT + inverse and DCT-2/DCT-3 round trip, normal inputs."""
    rng = np.random.default_rng(2)
    dims = (2048, 2048)
    x = rng.standard_normal(dims).astype(np.float32 if single else np.float64)
    for op in ("realdft", "dct2", "dct3", "dst2", "dst3"):
        err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
        assert err <= tolerance(single, dims), (op, err)
    z = make_input("invrealdft", dims, rng, single, dist="normal")
    err = rel_l2(gpu_apply("invrealdft", z, dims, single), expected("invrealdft", z, dims))
    assert err <= tolerance(single, dims)


@pytest.mark.slow
def test_config_batched_4096_c128():
    """1024 independent complex DFTs of length 4096 (forward and inverse)."""
    rng = np.random.default_rng(1)
    eng = minfft_b200.engine(False)
    n, howmany = 4096, 1024
    x = (rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n))).astype(np.complex128)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty_like(xt)
    zt = torch.empty_like(xt)
    p = eng.plan("dft", (n,))
    p.batch("dft", xt.data_ptr(), yt.data_ptr(), howmany)
    p.batch("invdft", yt.data_ptr(), zt.data_ptr(), howmany)
    torch.cuda.synchronize()
    p.free()
    lib = oracle.library(oracle_kind(), False)
    aux = lib.mkaux("dft", (n,))
    ref = np.empty_like(x)
    for i in range(howmany):
        row = np.ascontiguousarray(x[i])
        lib.run("dft", row.ctypes.data, ref[i].ctypes.data, aux)
    lib.free(aux)
    assert rel_l2(yt.cpu().numpy(), ref) <= 1e-13
    assert rel_l2(zt.cpu().numpy() / n, x) <= 1e-13


@pytest.mark.slow
def test_config_3d_256_c64():
    rng = np.random.default_rng(3)
    dims = (256, 256, 256)
    x = make_input("dft", dims, rng, True)
    err = rel_l2(gpu_apply("dft", x, dims, True), expected("dft", x, dims))
    assert err <= tolerance(True, dims), err


@pytest.mark.slow
@pytest.mark.parametrize("single", [False, True], ids=["c128", "c64"])
def test_config_large_dft_2_26(single):
    rng = np.random.default_rng(5)
    dims = (1 << 26,)
    x = make_input("dft", dims, rng, single)
    err = rel_l2(gpu_apply("dft", x, dims, single), expected("dft", x, dims))
    assert err <= tolerance(single, dims), err


@pytest.mark.slow
@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_config_large_t4_2_24(single):
    rng = np.random.default_rng(6)
    dims = (1 << 24,)
    for op in ("dct4", "dst4"):
        x = make_input(op, dims, rng, single)
        err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
        assert err <= tolerance(single, dims), (op, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_autotuned_plans_stay_correct(single, tmp_path):
    """The autotuner may pick either kernel form and any tile size; every
    choice must give the same results, and the table survives a save/load."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(41)
    for dims in [(2048,), (64, 1024), (1024, 8), (1 << 15,)]:
        for op in OPS:
            x = make_input(op, dims, rng, single)
            p = eng.plan(OP_FAMILY[op], dims)
            eng.autotune(p.aux, op, 1, 2)
            p.free()
            err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
            assert err <= tolerance(single, dims), (op, dims, err)
    n = eng.tune_size()
    assert n > 0
    path = str(tmp_path / "tune.txt")
    eng.tune_save(path)
    eng.tune_clear()
    assert eng.tune_size() == 0
    eng.tune_load(path)
    assert eng.tune_size() == n


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("pipe", [0, 1], ids=["tile", "pipelined"])
@pytest.mark.parametrize("radix", [8, 16])
def test_every_forced_configuration_is_correct(single, pipe, radix):
    """Both kernel forms, both per-thread radices, at every tile size
    (transforms per CTA), forced as the default configuration, on row and
    column passes of every transform kind, including the 1025 columns of a
    2-D real DFT."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(43)
    saved = eng.tune_size()
    try:
        eng.tune_clear()
        for cpb in (1, 2, 4, 8, 16, 64):
            eng.tune_set_default(pipe, cpb, radix)
            for dims in [(64, 512), (8, 2048), (1 << 14,), (16, 2048)]:
                for op in OPS:
                    x = make_input(op, dims, rng, single)
                    err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
                    assert err <= tolerance(single, dims), (op, dims, cpb, err)
    finally:
        eng.tune_set_default(-1, 0, 16)
    assert saved >= 0



@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_host_async_mode(single):
    """Host-async mode: calls on page-locked host arrays are ordered on the
    plan's stream and return at once; plans on their own streams run
    concurrently; after synchronizing, every output matches the oracle.
    Pageable arrays keep the synchronous behaviour."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(45)
    rdt, cdt = oracle.np_dtypes(single)
    dims = (256, 512)
    ops = [("realdft", "invrealdft"), ("dct2", "dct3")]
    plans, streams, jobs = [], [], []
    try:
        for first, second in ops:
            plan = eng.plan(OP_FAMILY[first], dims)
            st = torch.cuda.Stream()
            plan.set_stream(st.cuda_stream)
            plan.set_host_async(True)
            plans.append(plan)
            streams.append(st)
            x = make_input(first, dims, rng, single)
            _, _, s1, c1 = shapes(first, dims)
            _, _, s2, c2 = shapes(second, dims)
            tdt = lambda c: {np.float32: torch.float32, np.float64: torch.float64, np.complex64: torch.complex64,
                             np.complex128: torch.complex128}[cdt if c else rdt]  # noqa: E731
            hx = torch.from_numpy(x).pin_memory()
            h1 = torch.empty(s1, dtype=tdt(c1)).pin_memory()
            h2 = torch.empty(s2, dtype=tdt(c2)).pin_memory()
            jobs.append((plan, first, second, x, hx, h1, h2))
        for plan, first, second, x, hx, h1, h2 in jobs:
            plan(first, hx.data_ptr(), h1.data_ptr())
            plan(second, h1.data_ptr(), h2.data_ptr())
        for plan in plans:
            plan.synchronize()
        for plan, first, second, x, hx, h1, h2 in jobs:
            y1 = expected(first, x, dims)
            assert rel_l2(h1.numpy(), y1) <= tolerance(single, dims), first
            y2 = expected(second, y1.astype(cdt if np.iscomplexobj(y1) else rdt), dims)
            assert rel_l2(h2.numpy(), y2) <= 4 * tolerance(single, dims), second
        # pageable arrays in host-async mode: still synchronous
        plan, first, second, x = jobs[0][0], jobs[0][1], jobs[0][2], jobs[0][3]
        _, _, s1, c1 = shapes(first, dims)
        y = np.zeros(s1, dtype=cdt if c1 else rdt)
        plan(first, np.ascontiguousarray(x).ctypes.data, y.ctypes.data)
        assert rel_l2(y, expected(first, x, dims)) <= tolerance(single, dims)
    finally:
        for plan in plans:
            plan.free()
