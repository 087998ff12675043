"""The C ABI from a plain C program: include/sgd_b200.h compiles as strict C99
and C++11, and tests/c_caller.c, linked against the library, checks the
host-only geometry entry point and the error protocol (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

INC = os.path.join(ROOT, "include")


def _need(tool):
    if shutil.which(tool) is None:
        pytest.skip(f"{tool} not installed")


@pytest.mark.parametrize("compiler,flags", [("gcc", ["-x", "c", "-std=c99"]), ("g++", ["-x", "c++", "-std=c++11"])])
def test_header_compiles_strictly(tmp_path, compiler, flags):
    _need(compiler)
    src = tmp_path / "h.c"
    src.write_text('#include "sgd_b200.h"\nint main(void) { return 0; }\n')
    r = subprocess.run([compiler, *flags, "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", INC, "-c", str(src),
                        "-o", str(tmp_path / "h.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_caller_error_protocol(tmp_path):
    _need("gcc")
    from sgd_b200 import _lib
    assert os.path.exists(_lib.LIB_PATH), "library not built"
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "c_caller"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", INC,
                        os.path.join(ROOT, "tests", "c_caller.c"), "-o", str(exe), "-L", libdir, "-lnetwork",
                        f"-Wl,-rpath,{libdir}", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


def test_reference_style_cpp_caller_links(tmp_path):
    """A C++ caller written as the reference's own (global MatrixD and A_B1,
    the project/back_project calls of SGD.cu:176-187) compiles against
    reference_compat.h and links against the library; without a GPU the
    layer's constructor throws instead of returning."""
    _need("g++")
    from sgd_b200 import _lib
    csrc = os.path.join(ROOT, "sgd_b200", "csrc")
    cuda_inc = "/usr/local/cuda/include"
    if not os.path.isdir(cuda_inc):
        pytest.skip("CUDA headers not installed")
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include <cstdio>
#include "reference_compat.h"
int main() {
    const int nx = 8, ny = 8, np = 4, nu = 12;
    double ang[np] = {0.0, 0.5, 1.0, 1.5};
    try {
        A_B1 layer(nx, ny, np, nu, 1.0, 1.0, 1.0, 100.0, 50.0, ang, nullptr, nullptr);
        MatrixD vol(nx * ny, 1), proj(np * nu, 1);
        vol.allocateMemory();
        proj.allocateMemory();
        layer.project(vol, proj, 1.0);
        layer.back_project(vol, proj, 1.0);
        std::printf("ran\n");
    } catch (const std::exception& e) {
        std::printf("threw: %s\n", e.what());
    }
    return 0;
}
''')
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "caller"
    r = subprocess.run(["g++", "-std=c++17", "-I", csrc, "-I", cuda_inc, str(src), "-o", str(exe), "-L", libdir,
                        "-lnetwork", f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and (r.stdout.startswith("ran") or r.stdout.startswith("threw")), r.stdout + r.stderr
