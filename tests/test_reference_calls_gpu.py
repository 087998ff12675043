"""The reference's Python operators' calls, replayed against this library on
the GPU.

tests/golden/operator_calls.json holds what python/operators/operators.py of
the reference, run unmodified, binds and calls (symbol, declared argtypes and
restype, argument order, the 12/11-argument inits with per-view dz/drho,
A_SF_operator's 10-argument init, A_B1_3D_operator's 14-argument init and its
int restype for an unsigned long long return).  Each operator is replayed
here with exactly those declarations and arguments; its projections must
equal, bit for bit, those of sgd_b200.operators (the same entry points
behind this package's own wrappers), be non-trivial, and pass a dot-product
adjoint check where the layer is an adjoint pair.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden", "operator_calls.json")
CTYPES = {"c_int": ctypes.c_int, "c_double": ctypes.c_double, "c_void_p": ctypes.c_void_p,
          "LP_c_double": ctypes.POINTER(ctypes.c_double), None: None}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def ops():
    with open(GOLDEN) as f:
        return json.load(f)["operators"]


def bind(L, call):
    fn = getattr(L, call["symbol"])
    fn.argtypes = [CTYPES[t] for t in call["argtypes"]]
    fn.restype = CTYPES[call["restype"]]
    return fn


def ours(op):
    """The same operator through sgd_b200.operators."""
    from sgd_b200 import operators as so
    g, a = op["geometry"], {k: np.asarray(v) for k, v in op["arrays"].items()}
    kw = {"dz": a["dz"], "drho": a["drho"]} if op["offsets"] else {}
    if op["class"] in ("A_H0_operator", "A_Hl_operator"):
        return getattr(so, op["class"])(g["nx"], g["ny"], g["nnp"], g["nu"], g["dt"], g["du"], g["lsd"], g["lso"],
                                        a["angles"], **kw)
    if op["class"] == "A_B1_3D_operator":
        return so.A_B1_3D_operator(g["nx"], g["ny"], g["nz"], g["nnp"], g["nu"], g["nv"], g["dx"], g["dy"], g["dz"],
                                   g["du"], g["dv"], g["lsd"], g["lso"], a["angles"])
    return getattr(so, op["class"])(g["nx"], g["ny"], g["nnp"], g["nu"], g["dx"], g["dy"], g["du"], g["lsd"],
                                    g["lso"], a["angles"], **kw)


@pytest.mark.parametrize("idx", range(6))
def test_replayed_reference_calls_match_the_package(idx):
    from sgd_b200 import _lib
    op = ops()[idx]
    L = ctypes.CDLL(_lib.LIB_PATH)
    arrays = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in op["arrays"].items()}
    dp = ctypes.POINTER(ctypes.c_double)

    def args_of(call, extra):
        out = []
        for a in call["args"]:
            if isinstance(a, dict) and "array" in a:
                out.append((extra.get(a["array"]) if a["array"] in extra else arrays[a["array"]]).ctypes.data_as(dp))
            elif isinstance(a, dict) and a.get("handle"):
                out.append(handle)
            else:
                out.append(a)
        return out

    init, fwd, bwd = bind(L, op["init"]), bind(L, op["forward"]), bind(L, op["backward"])
    handle = init(*args_of(op["init"], {}))
    assert handle, _lib.last_error()
    m, n = op["shape"]
    rng = np.random.default_rng(idx)
    x = rng.random(n)
    y = np.zeros(m)
    fwd(*args_of(op["forward"], {"x": x, "y": y}))
    yin = rng.random(m)
    xt = np.zeros(n)
    bwd(*args_of(op["backward"], {"x": xt, "y": yin}))
    A = ours(op)
    assert np.count_nonzero(y) > 0.05 * m
    if op["class"] == "A_B1_3D_operator":
        # its forward sums in FP64 atomics: the same values to ~1e-16, not
        # always the same last bit after rounding to FP32
        np.testing.assert_allclose(y, A.matvec(x), rtol=1e-6, atol=0)
    else:
        assert np.array_equal(y, A.matvec(x))
    assert np.array_equal(xt, A.rmatvec(yin))
    if op["class"] not in ("A_H0_operator", "A_B1_3D_operator"):
        # adjoint pairs (not the reference's H0, whose back projection skips
        # bins its forward keeps, nor its A_B1_3D, whose backward drops the
        # forward's axial normalisation)
        lhs, rhs = float(np.dot(y, yin)), float(np.dot(x, xt))
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    destroy = getattr(L, op["init"]["symbol"].replace("_init", "_destroy"))
    destroy.argtypes = [ctypes.c_void_p]
    destroy.restype = None
    destroy(handle)
