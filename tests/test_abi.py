"""The C-ABI boundary, checked without a GPU: both engine libraries load,
export every function declared in include/*.h, and the makers reject bad
arguments before touching the device (reference minfft.c:1062-1064:
non-positive or non-power-of-two lengths give NULL)."""
import ctypes
import os
import re
import subprocess

import pytest

import minfft_b200
from minfft_b200 import ERROR_NAMES  # noqa: F401

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in ("minfft.h", "minfft_b200.h"):
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(minfft\w*)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_header_declares_reference_api():
    names = declared_functions()
    ref = {f"minfft_{t}" for t in ("dft", "invdft", "realdft", "invrealdft", "dct2", "dst2", "dct3", "dst3", "dct4",
                                   "dst4")}
    for fam in ("dft", "realdft", "t2t3", "t4"):
        ref |= {f"minfft_mkaux_{fam}{s}" for s in ("_1d", "_2d", "_3d", "")}
    ref.add("minfft_free_aux")
    assert len(ref) == 27
    assert ref <= names


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
def test_library_exports_every_declared_symbol(single):
    path = minfft_b200.LIB_PATHS[single]
    assert os.path.exists(path), "engine library not built"
    missing = declared_functions() - exported(path)
    assert not missing, missing


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
def test_library_loads_and_binds(single):
    eng = minfft_b200.engine(single)
    assert eng.single == single
    for op in minfft_b200.OPS:
        assert getattr(eng.lib, "minfft_" + op)


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
def test_makers_reject_bad_arguments_without_device(single):
    eng = minfft_b200.engine(single)
    eng.last_error()
    for fam in ("dft", "realdft", "t2t3", "t4"):
        for bad in (0, -1, 3, 6, 1000):
            assert eng.mkaux(fam, [bad]) == 0
            assert eng.last_error() == 1  # EINVAL
        assert eng.mkaux(fam, [8, 12]) == 0
        assert eng.last_error() == 1
        assert eng.mkaux(fam, [4, 4, 0]) == 0
        assert eng.last_error() == 1
        assert eng.mkaux_generic(fam, []) == 0
        assert eng.last_error() == 1
    eng.free(0)  # NULL is ignored


@pytest.mark.parametrize("single", [False, True], ids=["double", "single"])
def test_null_plan_is_an_error_not_a_crash(single):
    eng = minfft_b200.engine(single)
    eng.last_error()
    buf = (ctypes.c_double * 8)()
    eng.run("dft", ctypes.addressof(buf), ctypes.addressof(buf), 0)
    assert eng.last_error() == 1


def test_engine_refuses_to_load_without_library(tmp_path, monkeypatch):
    monkeypatch.setitem(minfft_b200.LIB_PATHS, False, str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        minfft_b200.Engine(False)


def test_compile_time_root_constants_are_exact():
    """The in-register butterflies use literal cos(pi*q/16) constants; check
    every literal against a 40-digit evaluation."""
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 40
    src = open(os.path.join(ROOT, "minfft_b200", "csrc", "common.cuh")).read()
    vals = re.findall(r"q == (\d) \? ([0-9.]+)", src)
    assert len(vals) == 7
    for q, v in vals:
        assert abs(mpmath.mpf(v) - mpmath.cos(mpmath.pi * int(q) / 16)) < 1e-30, (q, v)
