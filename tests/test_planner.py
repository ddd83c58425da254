"""Planner soundness on the CPU: every launch the engine would enqueue for a
shape stays inside its buffers, uses valid launch shapes, and never runs a
pass in place that cannot run in place.  This is the host-side reading of
the kernels' index arithmetic, done for every workload size before any of it
runs on a GPU."""
import itertools
import os
import re

import numpy as np
import pytest

import minfft_b200
from minfft_b200 import OPS

SHAPES = [(1,), (2,), (4,), (8,), (16,), (32,), (64,), (128,), (256,), (512,), (1024,), (2048,), (4096,), (8192,),
          (16384,), (32768,), (65536,), (1 << 17), (1 << 20), (4, 8), (16, 32), (1, 8), (8, 1), (64, 128), (2, 4, 8),
          (8, 16, 4), (2, 1, 4), (1, 2, 1), (2, 2, 4, 8), (32, 32, 32), (8192, 4), (4, 8192), (2, 16384), (16384, 2),
          (8, 8, 8192), (2048, 2048), (256, 256, 256), (1, 1, 1, 1, 2), (2, 8192, 2)]
SHAPES = [s if isinstance(s, tuple) else (s,) for s in SHAPES]
HUGE = [(1 << 26,), (1 << 24,), (1 << 22,), (4096, 4096), (16, 1 << 16)]


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
@pytest.mark.parametrize("dims", SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_plans_are_in_bounds(dims, single):
    eng = minfft_b200.engine(single)
    for op in OPS:
        for howmany, alias in itertools.product((1, 3), (False, True)):
            bad, rep, n = eng.plan_selfcheck(op, dims, howmany, alias)
            assert bad == 0, f"{op} {dims} howmany={howmany} alias={alias}:\n{rep}"
            assert n >= 1 or (op in ("dft", "invdft", "dct3", "dst3") and int(np.prod(dims)) == 1 and alias)


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
@pytest.mark.parametrize("dims", HUGE, ids=lambda d: "x".join(map(str, d)))
def test_workload_plans_are_in_bounds(dims, single):
    eng = minfft_b200.engine(single)
    for op in OPS:
        for alias in (False, True):
            bad, rep, _ = eng.plan_selfcheck(op, dims, 1, alias)
            assert bad == 0, f"{op} {dims} alias={alias}:\n{rep}"


def test_batched_4096_plan_is_one_launch_per_direction():
    eng = minfft_b200.engine(False)
    for op in ("dft", "invdft"):
        bad, rep, n = eng.plan_selfcheck(op, (4096,), 1024, False)
        assert bad == 0 and n == 1, rep


def test_2d_workload_launch_counts():
    """2048 x 2048: one fused row kernel and one column kernel per transform."""
    for single in (False, True):
        eng = minfft_b200.engine(single)
        for op in ("realdft", "invrealdft", "dct2", "dct3"):
            bad, rep, n = eng.plan_selfcheck(op, (2048, 2048), 1, False)
            assert bad == 0 and n == 2, (op, n, rep)


SPLIT_2D = [(1024, 32), (1024, 64), (2048, 2048), (4096, 32), (1024, 4096), (16384, 32)]


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
def test_split_column_real_dft_plans(single):
    """2-D real DFTs of >= 1024 rows split the column DFT into a radix-4 stage
    fused into the row pass and length-rows/4 column passes: two launches per
    direction, in bounds for single and batched calls, in place or not, and
    whatever tile size or radix the autotuner forces (the fused row passes
    keep four rows per CTA)."""
    eng = minfft_b200.engine(single)
    try:
        for forced in ((-1, 0, 16), (0, 1, 16), (0, 8, 8), (0, 32, 16), (1, 4, 16)):
            eng.tune_set_default(*forced)
            for dims in SPLIT_2D:
                for op in ("realdft", "invrealdft"):
                    for howmany in (1, 3):
                        for alias in (False, True):
                            bad, rep, n = eng.plan_selfcheck(op, dims, howmany, alias)
                            assert bad == 0, (forced, op, dims, howmany, alias, rep)
                            assert n == 2, (forced, op, dims, howmany, n)
        # below the row threshold, or rows too short for four per CTA: the plain plan
        eng.tune_set_default(-1, 0)
        for dims in ((512, 64), (2048, 16)):
            bad, rep, n = eng.plan_selfcheck("realdft", dims, 1, False)
            assert bad == 0 and n == 2, (dims, n, rep)
    finally:
        eng.tune_set_default(-1, 0)


def test_selfcheck_rejects_bad_arguments():
    eng = minfft_b200.engine(False)
    assert eng.plan_selfcheck("dft", (12,))[0] == -1
    assert eng.plan_selfcheck("dft", (8,), howmany=0)[0] == -1


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
@pytest.mark.parametrize("pipe", [0, 1], ids=["tile", "pipelined"])
@pytest.mark.parametrize("radix", [8, 16])
def test_every_launch_configuration_is_in_bounds(single, pipe, radix):
    """Every kernel form, radix and tile size the autotuner may pick, on every shape."""
    eng = minfft_b200.engine(single)
    try:
        for cpb in (1, 2, 4, 8, 16, 32, 64, 128, 256, 512):
            eng.tune_set_default(pipe, cpb, radix)
            for dims in SHAPES + HUGE[:3]:
                for op in OPS:
                    for alias in (False, True):
                        bad, rep, _ = eng.plan_selfcheck(op, dims, 2, alias)
                        assert bad == 0, f"pipe={pipe} cpb={cpb} {op} {dims} alias={alias}:\n{rep}"
    finally:
        eng.tune_set_default(-1, 0)


TC_SHAPES = [(256,), (4, 256), (256, 2), (256, 256), (256, 256, 256), (64, 64, 256), (256, 16, 4), (65536, 2),
             (1 << 16,), (1 << 24,), (2, 256, 2), (1 << 13,), (1 << 20,), (1 << 25,), (1 << 26,), (1 << 17, 4)]


@pytest.mark.parametrize("precision", ["tc_f16", "tc_bf16"])
@pytest.mark.parametrize("dims", TC_SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_tensor_core_plans_are_in_bounds(dims, precision):
    """The tensor-core passes replace every complex 256-point axis pass, the
    pre-twiddled passes of Stockham chains over HBM included (a chain in a
    tensor-core mode is split into as many 256-point passes as its pass count
    allows, plus one for the two-pass chains of 2^17 .. 2^24 points, which
    otherwise would have none); the plans stay sound."""
    eng = minfft_b200.engine(True)
    for op in OPS:
        for howmany, alias in itertools.product((1, 3), (False, True)):
            bad, rep, n = eng.plan_selfcheck(op, dims, howmany, alias, precision=precision)
            assert bad == 0, f"{op} {dims} {precision} howmany={howmany} alias={alias}:\n{rep}"
            _, _, n32 = eng.plan_selfcheck(op, dims, howmany, alias)
            # FP32 fuses the type-4 rotations of a 1-D chain into its first and
            # last passes; the tensor-core chains keep them as element-wise steps
            extra = 2 if op in ("dct4", "dst4") else 0
            assert n32 <= n <= n32 + 1 + extra


# (length, passes of its chain in a tensor-core mode: 256-point tensor-core
# passes first, then the CUDA-core ones, with the same pass count as FP32
# where that count allows a 256-point pass, else one more)
TC_CHAINS = [(1 << 16, ["tc:256", "tc:256"]), (1 << 20, ["tc:256", "cplx:4096"]),
             (1 << 24, ["tc:256", "tc:256", "tc:256"]), (1 << 25, ["tc:256", "tc:256", "cplx:512"]),
             (1 << 26, ["tc:256", "tc:256", "cplx:1024"]), (1 << 29, ["tc:256", "cplx:2048", "cplx:1024"])]


def chain_passes(report):
    out = []
    for lab in report.splitlines():
        m = re.search(r"(tc_pass|tc_stream|axis_pass|axis_pipe|stream_pass)<([a-z0-9+]+)?[^,]*,L=(\d+)", lab)
        if m:
            out.append(("tc" if m.group(1) in ("tc_pass", "tc_stream") else m.group(2)) + ":" + m.group(3))
    return out


@pytest.mark.parametrize("precision", ["tc_f16", "tc_bf16"])
@pytest.mark.parametrize("n,passes", TC_CHAINS, ids=[str(n) for n, _ in TC_CHAINS])
def test_tensor_core_chain_split(n, passes, precision):
    """A long complex axis in a tensor-core mode is split into as many
    256-point passes as its pass count (passes of up to 4096 points) allows,
    placed first; where that count allows none (2^24 in two passes), one more
    pass is taken.  The FP32 chain caps its passes at 1024 points, so it has
    as many passes for these lengths."""
    eng = minfft_b200.engine(True)
    bad, rep, _ = eng.plan_selfcheck("dft", (n,), 1, False, precision=precision)
    assert bad == 0, rep
    assert chain_passes(rep) == passes, rep
    bad, rep32, _ = eng.plan_selfcheck("dft", (n,), 1, False)
    assert bad == 0 and len(chain_passes(rep32)) == len(passes) and "tc_" not in rep32, rep32
    assert all(int(p.split(":")[1]) <= 1024 for p in chain_passes(rep32)), rep32


def test_tensor_core_modes_need_the_single_library():
    eng = minfft_b200.engine(False)
    bad, _, _ = eng.plan_selfcheck("dft", (256,), 1, False, precision="tc_f16")
    assert bad == -1


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_tuning_table_file_round_trip(single):
    """The autotuner's table saves to and loads from a text file: comment
    lines and malformed lines are skipped, entries with a radix other than 8
    or 16 are dropped, and a saved table reloads to the same entries.  Plans
    stay sound with a loaded table, also when an entry for one of their
    launches holds values outside the launch's limits (every tuned value is
    checked before use)."""
    eng = minfft_b200.engine(single)
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "tune")  # git-ignored
    os.makedirs(d, exist_ok=True)
    tag = "f32" if single else "f64"
    src, out = os.path.join(d, f"in_{tag}.txt"), os.path.join(d, f"out_{tag}.txt")
    good = ["0 4096 0 0 1 1 1 1 1 0 1 8", "0 512 1 0 0 4100 1 1025 1025 1 4 16", "3 1024 0 0 1 2048 1 1 1 0 2 16",
            "0 4096 0 0 1 8 1 1 1 0 100000 16"]
    with open(src, "w") as f:
        f.write("# a comment\n" + "\n".join(good) + "\nnot a line\n0 4096 0 0 1 1 1 1 1 0 1 4\n1 2 3\n")
    try:
        eng.tune_clear()
        eng.tune_load(src)
        assert eng.tune_size() == len(good)
        eng.tune_save(out)
        with open(out) as f:
            saved = [ln.strip() for ln in f if ln.strip() and not ln.startswith("#")]
        assert sorted(saved) == sorted(good)
        for op, dims in (("dft", (4096,)), ("dft", (2048, 2048)), ("realdft", (2048, 2048)), ("dct2", (1024,))):
            bad, rep, _ = eng.plan_selfcheck(op, dims, 1, False)
            assert bad == 0, rep
        eng.tune_clear()
        assert eng.tune_size() == 0
        # the key of the one 4096-point row launch (complex, L, row mode, no
        # pre-twiddle, staged or not, batch 1, unit strides): a valid entry
        # is used (the pipelined form), out-of-range values are refused at
        # planning time and the planner's own choice stays
        with open(src, "w") as f:
            f.write("0 4096 0 0 0 1 1 1 1 1 1 16\n0 4096 0 0 1 1 1 1 1 1 1 16\n")
        eng.tune_load(src)
        bad, rep, _ = eng.plan_selfcheck("dft", (4096,), 1, False)
        assert bad == 0 and rep.startswith("axis_pipe<cplx,L=4096,row>"), rep
        for form, cpb, radix in ((0, 100000, 16), (1, 100000, 8), (0, 0, 16), (1, -5, 16), (0, 3, 8)):
            with open(src, "w") as f:
                for staged in (0, 1):
                    f.write(f"0 4096 0 0 {staged} 1 1 1 1 {form} {cpb} {radix}\n")
            eng.tune_clear()
            eng.tune_load(src)
            assert eng.tune_size() == 2
            bad, rep, n = eng.plan_selfcheck("dft", (4096,), 1, False)
            assert bad == 0 and n == 1 and rep.startswith("axis_pass<cplx,L=4096,row>"), (form, cpb, radix, rep)
    finally:
        eng.tune_clear()


@pytest.mark.parametrize("precision", ["tc_f16", "tc_bf16"])
def test_tensor_core_type4_chain(precision):
    """The half-length chain of a 2^24-point DCT-4 (2^23 points) runs two
    256-point tensor-core passes in a tensor-core mode; the last pass, on the
    CUDA cores, takes the post-rotation into its store, and the pre-rotation
    stays a separate element-wise step before the tensor-core pass."""
    eng = minfft_b200.engine(True)
    bad, rep, _ = eng.plan_selfcheck("dct4", (1 << 24,), 1, False, precision=precision)
    assert bad == 0, rep
    assert chain_passes(rep) == ["tc:256", "tc:256", "cplx+t4post:128"], rep
    labs = rep.splitlines()
    assert any("line<t4_pre>" in lab for lab in labs), rep
    assert not any("line<t4_post>" in lab for lab in labs), rep
    # a last pass longer than 1024 points (2^19 = 256 x 2048) keeps the
    # post-rotation as an element-wise step
    bad, rep, _ = eng.plan_selfcheck("dct4", (1 << 20,), 1, False, precision=precision)
    assert bad == 0, rep
    assert chain_passes(rep) == ["tc:256", "cplx:2048"], rep
    labs = rep.splitlines()
    assert any("line<t4_pre>" in lab for lab in labs) and any("line<t4_post>" in lab for lab in labs), rep


@pytest.mark.parametrize("precision", ["fp32", "tc_f16", "tc_bf16"])
def test_fused_type4_pass_lengths(precision):
    """Every 1-D type-4 chain, in every precision mode, fuses its rotations
    only into passes of 128 to 1024 points, and each rotation is done exactly
    once: fused into an end pass or as its element-wise step."""
    eng = minfft_b200.engine(True)
    for b in range(13, 28):
        bad, rep, _ = eng.plan_selfcheck("dct4", (1 << b,), 1, False, precision=precision)
        assert bad == 0, rep
        fused = re.findall(r"(t4pre\+cplx|cplx\+t4post),L=(\d+)", rep)
        assert all(128 <= int(L) <= 1024 for _, L in fused), (b, rep)
        kinds = [k for k, _ in fused]
        if "line<" in rep or kinds:  # a chain (shorter lines run in one CTA)
            assert kinds.count("t4pre+cplx") + rep.count("line<t4_pre>") == 1, (b, rep)
            assert kinds.count("cplx+t4post") + rep.count("line<t4_post>") == 1, (b, rep)
