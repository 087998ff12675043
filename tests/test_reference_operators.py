"""The reference's own Python operators (python/operators/operators.py) as
callers of this library, on the CPU.

tests/golden/operator_calls.json records, from that module run unmodified,
which symbols it binds, the argtypes and restypes it declares and how it
calls them (tests/golden/make_operator_calls.py); test_reference_calls_gpu.py
replays it on a GPU.  Here: the record is current with the module (when the
reference tree is present), every symbol it binds is exported by the library
and declared in include/sgd_b200.h with the same number of parameters, and
the unmodified module driving the real library without a GPU gets a clean
failure (a null handle and -1 returns), not a crash.
"""
import ctypes
import json
import os
import re
import sys

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
import make_operator_calls as moc  # noqa: E402

REF = moc.default_reference()
HAVE_REF = os.path.exists(os.path.join(REF, "python", "operators", "operators.py"))


def fixture():
    with open(moc.OUT) as f:
        return json.load(f)


@pytest.mark.skipif(not HAVE_REF, reason="reference tree not present")
def test_record_is_current():
    mod = moc.load_reference_module(REF)
    assert json.loads(json.dumps(moc.record(mod))) == fixture()["operators"]


def _header_params():
    """Parameter count of each function declared in include/sgd_b200.h."""
    text = open(os.path.join(ROOT, "include", "sgd_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_every_bound_symbol_is_exported_and_declared():
    from sgd_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    decl = _header_params()
    for op in fixture()["operators"]:
        for what in ("init", "forward", "backward"):
            call = op[what]
            getattr(L, call["symbol"])  # raises AttributeError when missing
            assert call["symbol"] in decl, call["symbol"]
            assert len(call["argtypes"]) == decl[call["symbol"]] == len(call["args"]), (call["symbol"], call)


@pytest.mark.skipif(not HAVE_REF, reason="reference tree not present")
def test_unmodified_module_against_the_library_fails_cleanly_without_gpu(tmp_path):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: test_reference_calls_gpu.py covers this")
    from sgd_b200 import _lib
    build = tmp_path / "build"
    build.mkdir()
    os.symlink(_lib.LIB_PATH, build / "libnetwork.so")
    work = tmp_path / "run"
    work.mkdir()
    mod = moc.load_reference_module(REF)
    cwd = os.getcwd()
    os.chdir(work)  # the module loads '../build/libnetwork.so'
    try:
        n = 8
        ang = 2 * np.pi * np.arange(n) / n
        A = mod.A_B1_operator(16, 16, n, 24, 1.0, 1.0, 1.0, 100.0, 50.0, ang, dz=np.zeros(n), drho=np.zeros(n))
        assert not A.cpointer  # b1_init: NULL, no device
        y = A.matvec(np.ones(16 * 16))
        assert y.shape == (n * 24,) and not y.any()
        assert _lib.last_error()
    finally:
        os.chdir(cwd)
