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
