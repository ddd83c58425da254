"""The CPU oracle (restatement of reference minfft.c) against the golden
vectors produced by the compiled reference, and against the compiled
reference directly where oracle/_ref was built."""
import os

import numpy as np
import pytest

import oracle
from conftest import rel_l2
from minfft_b200._abi import OPS, shapes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases(single):
    data = np.load(os.path.join(GOLDEN, "golden_f32.npz" if single else "golden_f64.npz"))
    cases = {}
    for k in data.files:
        op, dims, what = k.split("|")
        cases.setdefault((op, dims), {})[what] = data[k]
    return [(op, tuple(int(v) for v in dims.split("x")), d["in"], d["out"]) for (op, dims), d in sorted(cases.items())]


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_restatement_matches_reference_golden(single):
    worst = 0.0
    tol = 2e-7 if single else 1e-15
    for op, dims, x, y in golden_cases(single):
        got = oracle.apply(op, x, dims, single=single, kind="restatement")
        assert got.shape == y.shape, (op, dims)
        err = rel_l2(got, y)
        worst = max(worst, err)
        assert err <= tol, (op, dims, err)
    assert worst > 0 or not single  # the single build really is a different precision


def test_golden_covers_every_transform_and_edge_size():
    cases = golden_cases(False)
    ops = {c[0] for c in cases}
    assert ops == set(OPS)
    dims = {c[1] for c in cases}
    for n in (1, 2, 4, 8, 16):
        assert (n,) in dims
    assert any(1 in d and len(d) > 1 for d in dims)


@pytest.mark.skipif(not oracle.available("reference"), reason="compiled reference not built here")
@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_restatement_matches_compiled_reference(single):
    rng = np.random.default_rng(7)
    tol = 2e-7 if single else 1e-15
    for dims in [(4096,), (64, 128), (8, 16, 32)]:
        for op in OPS:
            ins, inc, _, _ = shapes(op, dims)
            x = rng.standard_normal(ins) + (1j * rng.standard_normal(ins) if inc else 0)
            a = oracle.apply(op, x, dims, single=single, kind="restatement")
            b = oracle.apply(op, x, dims, single=single, kind="reference")
            assert rel_l2(a, b) <= tol, (op, dims)


def test_reference_definitions_match_scipy():
    """Second opinion: the double oracle equals the FFTW-compatible
    definitions (reference README "Transforms") as computed by scipy.fft."""
    sf = pytest.importorskip("scipy.fft")
    rng = np.random.default_rng(3)
    for dims in [(64,), (16, 32), (4, 8, 16)]:
        xc = rng.standard_normal(dims) + 1j * rng.standard_normal(dims)
        xr = rng.standard_normal(dims)
        n = int(np.prod(dims))
        assert rel_l2(oracle.apply("dft", xc, dims), sf.fftn(xc)) < 1e-14
        assert rel_l2(oracle.apply("invdft", xc, dims), sf.ifftn(xc) * n) < 1e-14
        assert rel_l2(oracle.apply("realdft", xr, dims), sf.rfftn(xr)) < 1e-14
        for t in (2, 3, 4):
            assert rel_l2(oracle.apply(f"dct{t}", xr, dims), sf.dctn(xr, type=t)) < 1e-14
            assert rel_l2(oracle.apply(f"dst{t}", xr, dims), sf.dstn(xr, type=t)) < 1e-14


def test_makers_reject_bad_sizes():
    lib = oracle.library("restatement")
    for fam in ("dft", "realdft", "t2t3", "t4"):
        for bad in (0, -4, 3, 12):
            assert lib.mkaux(fam, [bad]) == 0
        assert lib.mkaux(fam, [8, 6]) == 0
        assert lib.mkaux_generic(fam, []) == 0  # d < 1


def test_round_trip_scaling():
    """dft/invdft scale by N, realdft/invrealdft by N, dct2/dct3 by 2N,
    dct4/dct4 by 2N (per dimension), as documented in the reference README."""
    rng = np.random.default_rng(11)
    dims = (8, 16)
    n = 128
    xc = rng.standard_normal(dims) + 1j * rng.standard_normal(dims)
    xr = rng.standard_normal(dims)
    y = oracle.apply("invdft", oracle.apply("dft", xc, dims), dims)
    assert rel_l2(y / n, xc) < 1e-14
    y = oracle.apply("invrealdft", oracle.apply("realdft", xr, dims), dims)
    assert rel_l2(y / n, xr) < 1e-14
    y = oracle.apply("dct3", oracle.apply("dct2", xr, dims), dims)
    assert rel_l2(y / (4 * n), xr) < 1e-14
    y = oracle.apply("dct4", oracle.apply("dct4", xr, dims), dims)
    assert rel_l2(y / (4 * n), xr) < 1e-14
