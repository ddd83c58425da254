"""Full-size parity of the largest workloads against the FP64 oracle (the
compiled reference where it was built), through the C ABI.

* 256^3 complex DFT in c64 (uniform[-1,1) inputs): the plain FP32 path at the
  FP32 bar and both tensor-core split-precision modes at 1e-6, forward and
  inverse.
* 2^26-point complex DFT in c64: the same three arithmetic modes.
* 2^24-point DCT-4 and DST-4 in f32 in every mode.
* The 20000-transform mixed batch of the benchmark (log2 n uniform in 4..16,
  the eight forward kinds, f32, standard-normal inputs) as ONE autotuned
  launch, every job checked.

Each relative L2 error is printed (pytest -s shows them).  Reference:
minfft.c:77-272 (the DFT the tensor-core stages replace), :890-981 (type 4),
:287-981 (the caller loop the mixed batch replaces).
"""
import numpy as np
import pytest

import minfft_b200
import oracle
from conftest import rel_l2, tolerance
from minfft_b200 import shapes

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TC_BAR = 1e-6
MODES = ("fp32", "tc_f16", "tc_bf16")
_cache = {}


def bar(mode, dims):
    return tolerance(True, dims) if mode == "fp32" else TC_BAR


def uniform_c64(dims, seed):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, dims) + 1j * rng.uniform(-1, 1, dims)).astype(np.complex64)


def oracle_out(key, op, x, dims):
    """FP64 oracle result of op on x (upcast), cached across modes."""
    k = (key, op)
    if k not in _cache:
        xx = x.astype(np.complex128) if np.iscomplexobj(x) else x.astype(np.float64)
        _cache[k] = oracle.apply(op, xx, dims, single=False, kind=oracle.best_kind())
    return _cache[k]


def run_mode(family, op, x, dims, mode):
    eng = minfft_b200.engine(True)
    plan = eng.plan(family, dims)
    try:
        eng.set_precision(plan.aux, mode)
        if mode != "fp32":  # the tensor-core passes do run
            eng.profile(plan.aux, 1)
            probe = torch.zeros(2 * int(np.prod(dims)) + 8, dtype=torch.float32, device="cuda")
            out = torch.zeros_like(probe)
            plan(op, probe.data_ptr(), out.data_ptr())
            labels = [s[0] for s in eng.profile_stats(plan.aux)]
            eng.profile(plan.aux, 0)
            assert any(lab.startswith(("tc_pass<", "tc_stream<")) for lab in labels), labels
        xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        _, _, out_shape, out_c = shapes(op, dims)
        y = torch.full(out_shape, float("nan"), dtype=torch.complex64 if out_c else torch.float32, device="cuda")
        plan(op, xt.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        eng.tc_status(plan.aux)
        return y.cpu().numpy()
    finally:
        plan.free()


@pytest.mark.parametrize("mode", MODES)
def test_3d256_c64_every_mode_vs_oracle(mode):
    dims = (256, 256, 256)
    if "x3d" not in _cache:
        _cache["x3d"] = uniform_c64(dims, 3)
    x = _cache["x3d"]
    for op in ("dft", "invdft"):
        err = rel_l2(run_mode("dft", op, x, dims, mode), oracle_out("3d", op, x, dims))
        print(f"256^3 c64 {op} {mode}: rel L2 vs FP64 oracle {err:.3e}")
        assert err <= bar(mode, dims), (op, mode, err)


@pytest.mark.parametrize("mode", MODES)
def test_dft_2_26_c64_every_mode_vs_oracle(mode):
    dims = (1 << 26,)
    if "x26" not in _cache:
        _cache["x26"] = uniform_c64(dims, 5)
    x = _cache["x26"]
    for op in ("dft", "invdft"):
        err = rel_l2(run_mode("dft", op, x, dims, mode), oracle_out("26", op, x, dims))
        print(f"2^26 c64 {op} {mode}: rel L2 vs FP64 oracle {err:.3e}")
        assert err <= bar(mode, dims), (op, mode, err)


@pytest.mark.parametrize("mode", MODES)
def test_t4_2_24_f32_every_mode_vs_oracle(mode):
    dims = (1 << 24,)
    if "r24" not in _cache:
        _cache["r24"] = np.random.default_rng(6).uniform(-1, 1, dims).astype(np.float32)
    x = _cache["r24"]
    for op in ("dct4", "dst4"):
        err = rel_l2(run_mode("t4", op, x, dims, mode), oracle_out("t4", op, x, dims))
        print(f"2^24 f32 {op} {mode}: rel L2 vs FP64 oracle {err:.3e}")
        assert err <= bar(mode, dims), (op, mode, err)


def mixed_jobs():
    """The benchmark's 20000-job list: the same seed and draws."""
    kinds = ("dft", "realdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4")
    rng = np.random.default_rng(4)
    ops = [kinds[k] for k in rng.integers(0, len(kinds), 20000)]
    ns = [1 << int(v) for v in rng.integers(4, 17, 20000)]
    return ops, ns


def test_mixed_20000_one_launch_every_job_vs_oracle():
    ops, ns = mixed_jobs()
    eng = minfft_b200.engine(True)
    rng = np.random.default_rng(8)
    # one host image of every input (256-byte aligned slices), one upload
    offs, tot = [], 0
    for op, n in zip(ops, ns):
        ins, inc, outs, outc = shapes(op, (n,))
        bi = int(np.prod(ins)) * 4 * (2 if inc else 1)
        bo = int(np.prod(outs)) * 4 * (2 if outc else 1)
        offs.append((tot, bi, tot + (bi + 255) // 256 * 256, bo))
        tot = offs[-1][2] + (bo + 255) // 256 * 256
    image = np.zeros(tot // 4, dtype=np.float32)
    inputs = []
    for (oi, bi, _, _), op, n in zip(offs, ops, ns):
        v = rng.standard_normal(bi // 4).astype(np.float32)
        image[oi // 4: oi // 4 + bi // 4] = v
        ins, inc, _, _ = shapes(op, (n,))
        inputs.append(v.view(np.complex64).reshape(ins) if inc else v.reshape(ins))
    pool = torch.from_numpy(image).cuda()
    base = pool.data_ptr()
    h = eng.mixed_plan([(op, n, base + oi, base + oo) for (oi, _, oo, _), op, n in zip(offs, ops, ns)])
    try:
        eng.mixed_autotune(h, 1)
        pool.copy_(torch.from_numpy(image))  # autotuning ran the batch: restore the inputs
        eng.mixed_execute(h)
        torch.cuda.synchronize()
        out = pool.cpu().numpy()
    finally:
        eng.mixed_free(h)
    groups = {}
    for i, (op, n) in enumerate(zip(ops, ns)):
        groups.setdefault((op, n), []).append(i)
    worst = 0.0
    for (op, n), idx in sorted(groups.items()):
        _, _, outs, outc = shapes(op, (n,))
        rows = [inputs[i].astype(np.complex128 if np.iscomplexobj(inputs[i]) else np.float64) for i in idx]
        refs = oracle.apply_rows(op, rows, n, single=False, kind=oracle.best_kind())
        for i, ref in zip(idx, refs):
            oo, bo = offs[i][2], offs[i][3]
            got = out[oo // 4: oo // 4 + bo // 4]
            got = got.view(np.complex64).reshape(outs) if outc else got.reshape(outs)
            err = rel_l2(got, ref)
            worst = max(worst, err / tolerance(True, (n,)))
            assert err <= tolerance(True, (n,)), (i, op, n, err)
    print(f"mixed 20000: all {len(ops)} jobs within the FP32 bar; worst error / bar = {worst:.3f}")
