"""Mixed batches (minfft_b200_mixed_*): many independent 1-D transforms of
every kind and length in one persistent, graph-launched kernel, each checked
against the double-precision oracle; plus the error paths of the planner."""
import numpy as np
import pytest

import minfft_b200
import oracle
from conftest import rel_l2, tolerance
from minfft_b200 import shapes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

OPS8 = ("dft", "realdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4")


class Pool:
    """One device allocation carved into 256-byte aligned slices."""

    def __init__(self, nbytes):
        self.buf = torch.zeros(nbytes // 8 + 64, dtype=torch.float64, device="cuda")
        self.base = self.buf.data_ptr()
        self.off = 0

    def take(self, nbytes):
        p = self.base + self.off
        self.off += (nbytes + 255) // 256 * 256
        assert self.off <= self.buf.numel() * 8
        return p


def make_batch(single, specs, rng):
    rdt, cdt = oracle.np_dtypes(single)
    total = 0
    for op, n in specs:
        ins, inc, outs, outc = shapes(op, (n,))
        total += (int(np.prod(ins)) * (np.dtype(cdt if inc else rdt).itemsize) + 256)
        total += (int(np.prod(outs)) * (np.dtype(cdt if outc else rdt).itemsize) + 256)
    pool = Pool(total + 4096)
    jobs, host = [], []
    for op, n in specs:
        ins, inc, outs, outc = shapes(op, (n,))
        x = rng.standard_normal(ins)
        if inc:
            x = x + 1j * rng.standard_normal(ins)
        x = x.astype(cdt if inc else rdt)
        ip = pool.take(x.nbytes)
        onb = int(np.prod(outs)) * np.dtype(cdt if outc else rdt).itemsize
        opp = pool.take(onb)
        tin = torch.from_numpy(x.view(np.uint8).ravel()).cuda()
        pool.buf.view(torch.uint8)[ip - pool.base: ip - pool.base + x.nbytes].copy_(tin)
        jobs.append((op, n, ip, opp))
        host.append((op, n, x, opp - pool.base, onb, outs, cdt if outc else rdt))
    return pool, jobs, host


def check_batch(single, pool, host):
    raw = pool.buf.view(torch.uint8).cpu().numpy()
    for op, n, x, off, onb, outs, dt in host:
        got = raw[off: off + onb].view(dt).reshape(outs)
        ref = oracle.apply(op, x.astype(np.complex128 if np.iscomplexobj(x) else np.float64), (n,),
                           kind=oracle.best_kind())
        err = rel_l2(got, ref)
        assert err <= tolerance(single, (n,)), (op, n, err)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_mixed_batch_every_kind_and_length(single):
    rng = np.random.default_rng(7)
    specs = []
    for op in minfft_b200.OPS:
        for lg in (0, 1, 2, 3, 4, 6, 9, 12, 13, 14, 15, 16):
            specs.append((op, 1 << lg))
        if op not in ("dft", "invdft"):
            specs.append((op, 1 << 17))  # real lengths up to 131072
    specs += [("dct2", 256)] * 40 + [("dft", 64)] * 70  # groups split into several items
    eng = minfft_b200.engine(single)
    pool, jobs, host = make_batch(single, specs, rng)
    h = eng.mixed_plan(jobs)
    try:
        assert eng.mixed_items(h) >= len(minfft_b200.OPS)
        eng.mixed_execute(h)
        torch.cuda.synchronize()
        check_batch(single, pool, host)
        # relaunching the captured graph gives the same results
        snap = pool.buf.clone()
        eng.mixed_execute(h)
        torch.cuda.synchronize()
        assert torch.equal(snap, pool.buf)
    finally:
        eng.mixed_free(h)


def test_mixed_config_like_batch_after_autotune():
    """A scaled-down copy of the 20000-transform workload (log2 n uniform in
    4..16, the eight forward kinds, f32), autotuned, then checked."""
    rng = np.random.default_rng(11)
    specs = [(OPS8[rng.integers(0, 8)], 1 << int(rng.integers(4, 17))) for _ in range(600)]
    eng = minfft_b200.engine(True)
    pool, jobs, host = make_batch(True, specs, rng)
    h = eng.mixed_plan(jobs)
    try:
        eng.mixed_autotune(h, 1)
        eng.mixed_execute(h)
        torch.cuda.synchronize()
        check_batch(True, pool, host)
    finally:
        eng.mixed_free(h)


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_mixed_plan_rejects_bad_jobs(single):
    eng = minfft_b200.engine(single)
    buf = torch.zeros(1 << 20, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    bad = [
        [("dft", 12, p, p + 4096)],          # not a power of two
        [("dft", 1 << 17, p, p + 4096)],     # complex longer than 65536
        [("dct2", 1 << 18, p, p + 4096)],    # real longer than 131072
        [("dft", 64, p + 4, p + 4096)],      # misaligned complex input
        [(42, 64, p, p + 4096)],             # unknown transform
        [("dft", 64, 0, p)],                 # NULL pointer
    ]
    for jobs in bad:
        with pytest.raises(minfft_b200.MinfftError) as e:
            eng.mixed_plan(jobs)
        assert e.value.code == 1


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_mixed_cluster_form_every_long_kind(single, monkeypatch):
    """The cluster form of the long items (2^14 .. 2^16 complex points on
    eight CTAs in distributed shared memory, MINFFT_B200_MIXED_CLUSTER=1):
    every kind and long length, mixed with short items, against the oracle."""
    monkeypatch.setenv("MINFFT_B200_MIXED_CLUSTER", "1")
    rng = np.random.default_rng(17)
    specs = []
    for op in minfft_b200.OPS:
        lens = (14, 15, 16) if op in ("dft", "invdft") else (15, 16, 17)
        specs += [(op, 1 << lg) for lg in lens]
    specs += [("dct2", 256)] * 8 + [("dft", 64)] * 8 + [("dst4", 1 << 12)] * 4
    eng = minfft_b200.engine(single)
    pool, jobs, host = make_batch(single, specs, rng)
    h = eng.mixed_plan(jobs)
    try:
        eng.mixed_execute(h)
        torch.cuda.synchronize()
        check_batch(single, pool, host)
    finally:
        eng.mixed_free(h)


@pytest.mark.parametrize("cluster", ["0", "1"], ids=["scratch", "cluster"])
@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_mixed_long_items_only(single, cluster, monkeypatch):
    """A batch of long items and nothing else: every root table the long
    items read (the scratch form's two pass lengths, the cluster form's
    L/256- and 256-point DFTs) is built from the long items themselves, not
    borrowed from short items of those lengths."""
    monkeypatch.setenv("MINFFT_B200_MIXED_CLUSTER", cluster)
    rng = np.random.default_rng(23)
    specs = [("dft", 1 << 14)] * 3 + [("invdft", 1 << 15)] * 2 + [("dft", 1 << 16)] + [("realdft", 1 << 15)] + \
            [("dct2", 1 << 16)] + [("dst4", 1 << 17)]
    eng = minfft_b200.engine(single)
    pool, jobs, host = make_batch(single, specs, rng)
    h = eng.mixed_plan(jobs)
    try:
        eng.mixed_execute(h)
        torch.cuda.synchronize()
        check_batch(single, pool, host)
    finally:
        eng.mixed_free(h)
