"""The C-ABI library loads and exports every entry point include/*.h declares,
and its constructors reject bad geometry before their first CUDA call (no
compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            if m.group(1) not in ("if", "defined"):
                names.append(m.group(1))
    return names


def test_header_declares_reference_names():
    names = declared_functions()
    for n in ("b1_init", "b1_forward_projection", "b1_backward_projection", "sgd_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from sgd_b200 import _lib
    assert os.path.exists(_lib.LIB_PATH), "library not built"
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_library_binding_declares_types():
    from sgd_b200 import _lib
    L = _lib.lib()
    assert L.b1_init.restype is ctypes.c_void_p
    assert len(L.b1_init.argtypes) == 12


def test_operator_without_gpu_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import numpy as np
    from sgd_b200.operators import A_B1_operator
    from sgd_b200._lib import ProjectorError
    with pytest.raises(ProjectorError):
        A_B1_operator(8, 8, 4, 12, 1.0, 1.0, 1.0, 40.0, 20.0, np.linspace(0, 1, 4))


_NAN, _INF = float("nan"), float("inf")
_GEOMETRY_CHECKS = "pitches must be positive|lso < lsd|is not finite|angles pointer|invalid"


def _init(L, name, **over):
    """Calls constructor `name` on a small valid geometry with the arguments in
    `over` replaced: (handle, sgd_last_error())."""
    import numpy as np
    dp = ctypes.POINTER(ctypes.c_double)
    views = over.pop("views", np.linspace(0.0, 1.0, 4))
    a = dict(n=8, np=4, nu=12, d=1.0, du=1.0, lsd=40.0, lso=20.0, dz=None, drho=None)
    a.update(over)
    arrs = {k: None if a[k] is None else np.ascontiguousarray(a[k], dtype=np.float64) for k in ("dz", "drho")}
    views = np.ascontiguousarray(views, dtype=np.float64)
    ptr = lambda v: None if v is None else v.ctypes.data_as(dp)  # noqa: E731
    n, P, nu, d, du, lsd, lso = a["n"], a["np"], a["nu"], a["d"], a["du"], a["lsd"], a["lso"]
    if name in ("b1", "b0", "SF"):
        f = getattr(L, f"{name}_init")
        f.restype = ctypes.c_void_p
        f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [dp] * (3 if name != "SF" else 1)
        args = [n, n, P, nu, d, d, du, lsd, lso, ptr(views)]
        if name != "SF":
            args += [ptr(arrs["dz"]), ptr(arrs["drho"])]
        h = f(*args)
    elif name == "h0":
        L.h0_init.restype = ctypes.c_void_p
        L.h0_init.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 4 + [dp] * 3
        h = L.h0_init(n, n, P, nu, d, du, lsd, lso, ptr(views), ptr(arrs["dz"]), ptr(arrs["drho"]))
    elif name == "parallel":
        L.sgd_b0_parallel_init.restype = ctypes.c_void_p
        L.sgd_b0_parallel_init.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [dp]
        h = L.sgd_b0_parallel_init(n, n, P, nu, d, d, du, ptr(views))
    elif name in ("b1_3d", "sf3d"):
        f = L.sgd_b1_3d_init if name == "b1_3d" else L.sgd_sf3d_init
        f.restype = ctypes.c_void_p
        lead = [0] if name == "b1_3d" else [1, 0]
        f.argtypes = [ctypes.c_int] * (len(lead) + 6) + [ctypes.c_double] * 7 + [dp]
        h = f(*lead, n, n, n, P, nu, nu, d, d, a.get("dz_pitch", d), du, du, lsd, lso, ptr(views))
    else:
        raise KeyError(name)
    L.sgd_last_error.restype = ctypes.c_char_p
    return h, (L.sgd_last_error() or b"").decode()


def _destroy(L, name, h):
    if not h:
        return
    f = {"b1": "b1_destroy", "b0": "b0_destroy", "SF": "SF_destroy", "h0": "h0_destroy", "parallel": "b0_destroy",
         "b1_3d": "b1_3d_destroy", "sf3d": "sgd_sf3d_destroy"}[name]
    getattr(L, f).argtypes = [ctypes.c_void_p]
    getattr(L, f)(h)


_BAD = [
    ("nan angle", dict(views=[0.0, _NAN, 1.0, 2.0]), "angle of view 1 is not finite"),
    ("inf angle", dict(views=[0.0, 1.0, 2.0, _INF]), "angle of view 3 is not finite"),
    ("zero pitch", dict(d=0.0), "pitches must be positive and finite"),
    ("inf pitch", dict(d=_INF), "pitches must be positive and finite"),
    ("nan bin pitch", dict(du=_NAN), "pitches must be positive and finite"),
    ("lsd below lso", dict(lsd=10.0), "lso < lsd"),
    ("inf lsd", dict(lsd=_INF), "lso < lsd"),
    ("nan lso", dict(lso=_NAN), "lso < lsd"),
]
_FAN = ["b1", "b0", "SF", "h0"]


@pytest.mark.parametrize("name", _FAN + ["b1_3d", "sf3d", "parallel"])
@pytest.mark.parametrize("label,over,msg", _BAD, ids=[b[0] for b in _BAD])
def test_constructor_rejects_bad_geometry(name, label, over, msg):
    from sgd_b200 import _lib
    L = _lib.lib()
    if name == "parallel" and ("lso" in over or "lsd" in over):
        pytest.skip("parallel beam has no source distances")
    h, err = _init(L, name, **over)
    _destroy(L, name, h)
    assert not h, f"{name} accepted {label}"
    assert msg in err, err


@pytest.mark.parametrize("name", ["b1", "b0", "h0"])
@pytest.mark.parametrize("which", ["dz", "drho"])
def test_constructor_rejects_non_finite_view_offsets(name, which):
    from sgd_b200 import _lib
    L = _lib.lib()
    h, err = _init(L, name, **{which: [0.0, 0.0, _NAN, 0.0]})
    _destroy(L, name, h)
    assert not h and f"{which} of view 2 is not finite" in err, err


def test_cone_constructors_check_the_axial_pitch():
    from sgd_b200 import _lib
    L = _lib.lib()
    for name in ("b1_3d", "sf3d"):
        h, err = _init(L, name, dz_pitch=-1.0)
        _destroy(L, name, h)
        assert not h and "pitches must be positive" in err, err


@pytest.mark.parametrize("name", _FAN + ["b1_3d", "sf3d", "parallel"])
def test_valid_geometry_passes_the_checks(name):
    """A valid geometry gets past every check: without a GPU the constructor
    then fails at its first CUDA call, with a GPU it succeeds."""
    from sgd_b200 import _lib
    L = _lib.lib()
    h, err = _init(L, name, dz=[0.0, 0.5, -0.5, 1.0] if name in ("b1", "b0", "h0") else None,
                   drho=[0.0, 0.1, 0.2, 0.3] if name in ("b1", "b0", "h0") else None)
    _destroy(L, name, h)
    if not h:
        assert not re.search(_GEOMETRY_CHECKS, err), err


def test_bench_without_gpu_fails_loudly():
    """bench.py's own arm has no CPU fallback: without a GPU it exits non-zero
    and prints no result line."""
    import subprocess
    import sys
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([sys.executable, "bench.py", "--steps", "1", "--warmup", "1"], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode != 0
    assert not [line for line in r.stdout.splitlines() if line.startswith("{")]
