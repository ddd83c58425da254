"""The streamed column pass (persistent CTAs fed by tensor copies or
cp.async through an mbarrier pipeline, stream_pass.cuh) against the
double-precision oracle: forced as the default form, at every stage count
and both per-thread radices, on the column passes of 2-D and 3-D DFTs, the
split column DFT of 2-D real DFTs (1025 columns: a row pitch that is not a
multiple of 16 bytes in single precision, so the cp.async path), the passes
of Stockham chains over HBM (pre-twiddled, and the first pass with its
row-contiguous output), in-place calls and inputs offset from their
allocation (tensor copies refused, cp.async used)."""
import os

import numpy as np
import pytest

import minfft_b200
from conftest import rel_l2, tolerance
from test_gpu_parity import expected, gpu_apply, make_input

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(64, 512), (512, 16), (16, 64, 256), (256, 256), (2048, 2048), (1 << 16,), (1 << 20,), (32, 1024)]
OPS = ("dft", "invdft", "realdft", "invrealdft")


def labels(eng, op, dims):
    plan = eng.plan(minfft_b200.OP_FAMILY[op], dims)
    try:
        n = int(np.prod(dims))
        x = torch.zeros(n, dtype=torch.complex128, device="cuda")  # large enough in either precision
        y = torch.zeros(n, dtype=torch.complex128, device="cuda")
        eng.profile(plan.aux, 1)
        plan(op, x.data_ptr(), y.data_ptr())
        return [s[0] for s in eng.profile_stats(plan.aux)]
    finally:
        plan.free()


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("stages,radix", [(2, 16), (3, 16), (4, 8)])
def test_streamed_pass_matches_oracle(single, stages, radix):
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(61)
    try:
        eng.tune_clear()
        eng.tune_set_default(2, stages, radix)
        assert any("stream_pass" in lab for lab in labels(eng, "dft", (64, 512)))
        for dims in SHAPES:
            for op in OPS:
                x = make_input(op, dims, rng, single)
                err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
                assert err <= tolerance(single, dims), (op, dims, stages, radix, err)
        # in place
        dims = (256, 512)
        x = make_input("dft", dims, rng, single)
        err = rel_l2(gpu_apply("dft", x, dims, single, inplace=True), expected("dft", x, dims))
        assert err <= tolerance(single, dims)
    finally:
        eng.tune_set_default(-1, 0, 16)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_streamed_pass_with_offset_input(single):
    """An input that starts one complex element past a 16-byte boundary (f32)
    cannot be described by a tensor map; the pass copies with cp.async."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(62)
    dims = (128, 256)
    rdt, cdt = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    tdt = torch.complex64 if single else torch.complex128
    try:
        eng.tune_set_default(2, 3, 16)
        x = make_input("dft", dims, rng, single)
        buf = torch.zeros(x.size + 1, dtype=tdt, device="cuda")
        buf[1:] = torch.from_numpy(x.ravel()).cuda()
        y = torch.zeros(x.size, dtype=tdt, device="cuda")
        plan = eng.plan("dft", dims)
        try:
            esz = buf.element_size()
            plan("dft", buf.data_ptr() + esz, y.data_ptr())
            torch.cuda.synchronize()
        finally:
            plan.free()
        err = rel_l2(y.cpu().numpy().reshape(dims), expected("dft", x, dims))
        assert err <= tolerance(single, dims)
    finally:
        eng.tune_set_default(-1, 0, 16)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_fused_type4_chain_matches_oracle(single):
    """1-D DCT-4 / DST-4 lines longer than one CTA run their pre-rotation in
    the first pass over HBM and their post-rotation in the last one
    (LoadT4Chain, StoreT4Chain): single lines, several lines of a 2-D array,
    and in-place calls, against the oracle.  With MINFFT_B200_T4FUSE=0 the
    same cases run through the separate rotation line steps."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(63)
    fused = os.environ.get("MINFFT_B200_T4FUSE", "1") != "0"
    for dims in [(1 << 15,), (1 << 18,), (4, 1 << 16)]:
        plan_labels = labels(eng, "dct4", dims)
        if fused:
            assert any("t4pre" in lab for lab in plan_labels), plan_labels
        else:
            assert any("line<t4_pre>" in lab for lab in plan_labels), plan_labels
        for op in ("dct4", "dst4"):
            x = make_input(op, dims, rng, single)
            err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
            assert err <= tolerance(single, dims), (op, dims, err)
    dims = (1 << 16,)
    x = make_input("dst4", dims, rng, single)
    err = rel_l2(gpu_apply("dst4", x, dims, single, inplace=True), expected("dst4", x, dims))
    assert err <= tolerance(single, dims)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_fused_type4_chain_with_offset_arrays(single):
    """Real arrays that start one element past a complex boundary: the fused
    type-4 passes read and write their real pairs as two scalars instead of
    one vector (LoadT4Chain, StoreT4Chain), with the same results."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(64)
    tdt = torch.float32 if single else torch.float64
    for dims in [(1 << 17,), (2, 1 << 15)]:
        for op in ("dct4", "dst4"):
            x = make_input(op, dims, rng, single)
            n = x.size
            src = torch.zeros(n + 1, dtype=tdt, device="cuda")
            src[1:] = torch.from_numpy(x.ravel()).cuda()
            dst = torch.zeros(n + 1, dtype=tdt, device="cuda")
            plan = eng.plan("t4", dims)
            try:
                esz = src.element_size()
                plan(op, src.data_ptr() + esz, dst.data_ptr() + esz)
                torch.cuda.synchronize()
            finally:
                plan.free()
            err = rel_l2(dst[1:].cpu().numpy().reshape(dims), expected(op, x, dims))
            assert err <= tolerance(single, dims), (op, dims, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("form,cpb", [(3, 0), (3, 1), (4, 2), (4, 8)])
def test_streamed_rows_match_oracle(single, form, cpb):
    """The streamed row pass (bulk row copies into mbarrier stages, each
    kind's load stage reading the stage): forced as the default form (3: two
    stages, 4: three) for every transform kind, on rows of 2-D arrays (the
    split-column kinds of the 2048-row real DFT included), batches with a
    partial last tile, rows of odd byte length (the inverse real DFT's
    L+1 complex values in single precision: cp.async), in place."""
    eng = minfft_b200.engine(single)
    rng = np.random.default_rng(64)
    try:
        eng.tune_clear()
        eng.tune_set_default(form, cpb, 16)
        assert any("stream_rows" in lab for lab in labels(eng, "dct2", (64, 512)))
        for dims in [(64, 512), (4, 2048), (2048, 256), (2048, 2048), (4, 64, 128)]:
            for op in minfft_b200.OPS:
                x = make_input(op, dims, rng, single)
                err = rel_l2(gpu_apply(op, x, dims, single), expected(op, x, dims))
                assert err <= tolerance(single, dims), (op, dims, form, cpb, err)
        dims = (32, 1024)
        for op in ("realdft", "dct3"):
            x = make_input(op, dims, rng, single)
            err = rel_l2(gpu_apply(op, x, dims, single, inplace=True), expected(op, x, dims))
            assert err <= tolerance(single, dims), (op, "in place", err)
    finally:
        eng.tune_set_default(-1, 0, 16)
