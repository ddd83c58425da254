"""An unmodified C caller of the minfft API, built with gcc against the
engine's libraries.

tests/c_api/minfft_example.c uses only reference minfft.h: host arrays,
the plan makers, the ten transforms' families and minfft_free_aux, as the
reference README's "Interface" section shows.  It checks its results
against sums of the transform definitions and exits 0 (all checks pass),
1 (a result is off) or 2 (a plan maker returned NULL).

On CPU the program is built against the C restatement (oracle/) and the
compiled reference, both of which must pass: this checks the program itself.
It is also built against the engine's libraries, which must link, and,
without a GPU, must fail cleanly (makers return NULL).  On a GPU the program
built against the engine must pass every check, in double and in single
precision.
"""
import os
import shutil
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_api", "minfft_example.c")
OUT = os.path.join(ROOT, "tests", "c_api", "_build")
ENGINE_LIB = os.path.join(ROOT, "minfft_b200", "lib")

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")


def build(lib_path, single):
    """Compile the program against the shared library at lib_path."""
    os.makedirs(OUT, exist_ok=True)
    d, name = os.path.split(lib_path)
    exe = os.path.join(OUT, f"{os.path.splitext(name)[0]}_{int(single)}")
    cmd = ["gcc", "-O2", "-std=c99", "-Wall", "-Wextra", "-Werror", f"-DMINFFT_SINGLE={int(single)}", SRC,
           "-I", os.path.join(ROOT, "include"), "-L", d, f"-l:{name}", f"-Wl,-rpath,{d}", "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def run(exe):
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


def engine_lib(single):
    """The engine's in-tree library, as the other tests load it (built by
    `python -m minfft_b200.build`)."""
    path = os.path.join(ENGINE_LIB, "libminfft_b200_single.so" if single else "libminfft_b200.so")
    assert os.path.exists(path), f"{path} is missing: build it with `python -m minfft_b200.build`"
    return path


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("kind", ["restatement", "reference"])
def test_program_passes_against_the_cpu_libraries(kind, single):
    if kind == "reference" and not oracle.available("reference", single):
        oracle.build()
        if not oracle.available("reference", single):
            pytest.skip("the compiled reference is not available")
    oracle.library(kind, single)  # builds the restatement if needed
    rc, out = run(build(oracle._PATHS[(kind, single)], single))
    assert rc == 0, out
    assert out.count(" ok") == 8, out


@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_program_links_against_the_engine_and_fails_cleanly_without_a_gpu(single):
    exe = build(engine_lib(single), single)
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the gpu test runs the program")
    rc, out = run(exe)
    assert rc == 2 and "returned NULL" in out, out


@pytest.mark.gpu
@pytest.mark.parametrize("single", [False, True], ids=["f64", "f32"])
def test_program_passes_against_the_engine_on_a_gpu(single):
    rc, out = run(build(engine_lib(single), single))
    assert rc == 0, out
    assert out.count(" ok") == 8, out
