"""include/sfgpu.h from C and C++ callers (not ctypes).

The header must compile as C and as C++, and a C++ program that fills the
descriptors as an SFbox maintainer would (tests/abi/c1_residual.cpp) must
build against it and libsfgpu.so and, on a GPU, reproduce SFbox's own
residual for the C1 system (the fixture tests/golden/reference_cases.npz,
written by the reference's sources)."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "field_b200")
SRC = os.path.join(HERE, "abi", "c1_residual.cpp")


def test_header_compiles_as_c_and_cxx(tmp_path):
    for lang, comp in (("c", "gcc"), ("c++", "g++")):
        subprocess.run([comp, "-x", lang, "-fsyntax-only", "-Wall", "-Werror", "-pedantic", "-I", INC,
                        os.path.join(INC, "sfgpu.h")], check=True)


def _build(tmp_path):
    exe = str(tmp_path / "c1_residual")
    subprocess.run(["g++", "-O2", "-Wall", "-Werror", "-I", INC, SRC, "-L", LIBDIR, "-lsfgpu",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_cxx_caller_builds_against_the_library(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_cxx_caller_reproduces_sfbox_c1_residual(gpu_lib, tmp_path):
    exe = _build(tmp_path)
    with np.load(os.path.join(HERE, "golden", "reference_cases.npz")) as z:
        x, g, F = z["1d_flat_c1/x"], z["1d_flat_c1/g"], z["1d_flat_c1/F"][0]
    xf, ff = str(tmp_path / "x.bin"), str(tmp_path / "f.bin")
    x.astype("<f8").tofile(xf)
    r = subprocess.run([exe, xf, ff], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(ff, dtype="<f8")
    f, Fg = out[:-1], out[-1]
    assert f.size == g.size == 200
    assert np.max(np.abs(f - g)) <= 1e-12 * max(1.0, np.max(np.abs(g)))
    assert abs(Fg - F) <= 1e-12 * max(1.0, abs(F))
