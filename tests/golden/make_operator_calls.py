"""Records how the reference's Python operators (python/operators/operators.py,
run unmodified from the reference tree) bind and call the projector library:
for each operator class, the symbol each ctypes function is looked up by, the
argtypes and restype the module declares, and the arguments of its init,
forward and backward calls (scalars as passed; arrays by role).  Writes
tests/golden/operator_calls.json, which tests/test_reference_calls_gpu.py
replays against sgd_b200/libnetwork.so on a GPU (the reference tree is not
there) and tests/test_reference_operators.py regenerates and compares on the
CPU.

    python tests/golden/make_operator_calls.py [REFERENCE_ROOT]

REFERENCE_ROOT defaults to $SGD_REFERENCE, else the reference checkout beside
the repository.  pylops is not installed here: a stub providing
LinearOperator(dtype, shape) with matvec/rmatvec stands in for it (the module
only subclasses it).  The library is replaced by a recorder, so nothing is
computed.

Only the well-defined call forms are recorded: the 2D operators with per-view
dz/drho (12- and 11-argument inits), A_SF_operator and A_B1_3D_operator.  With
dz=None the module declares 10 (9 for H0/Hl) argtypes for an init whose C
signature has 12 (11): the last two pointer arguments are then whatever the
registers hold, in the reference's library as in this one.
"""
import ctypes
import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "operator_calls.json")


def stub_pylops():
    m = types.ModuleType("pylops")

    class LinearOperator:
        def __init__(self, dtype=None, shape=None, **kw):
            self.dtype = np.dtype(dtype)
            self.shape = tuple(shape)

        def matvec(self, x):
            return self._matvec(x)

        def rmatvec(self, y):
            return self._rmatvec(y)

    m.LinearOperator = LinearOperator
    return m


def load_reference_module(ref_root):
    sys.modules.setdefault("pylops", stub_pylops())
    path = os.path.join(ref_root, "python", "operators", "operators.py")
    spec = importlib.util.spec_from_file_location("reference_operators", path)
    mod = importlib.util.module_from_spec(spec)
    sys.dont_write_bytecode = True
    spec.loader.exec_module(mod)
    return mod


def _type_name(t):
    if t is None:
        return None
    return t.__name__


class _Fn:
    def __init__(self, log, name):
        self._log, self._name = log, name
        self.argtypes = None
        self.restype = ctypes.c_int

    def __call__(self, *args):
        self._log.append({"symbol": self._name, "argtypes": [_type_name(t) for t in (self.argtypes or [])],
                          "restype": _type_name(self.restype), "args": list(args)})
        if self.restype is ctypes.c_void_p:
            return 0xC0FFEE  # a stand-in handle
        return 0


class _Dll:
    def __init__(self, log):
        self._log, self._fns = log, {}

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return self._fns.setdefault(name, _Fn(self._log, name))


def _describe(arg, roles):
    """Scalar as is; a pointer by the role of the array it points at."""
    if isinstance(arg, (int, float)) and not isinstance(arg, bool):
        return arg
    if arg == 0xC0FFEE:
        return {"handle": True}
    addr = ctypes.cast(arg, ctypes.c_void_p).value
    for role, (lo, hi) in roles.items():
        if lo <= addr < hi:
            return {"array": role}
    return {"array": "?"}


def cases():
    """(operator class, its geometry, whether it is given per-view dz/drho)."""
    f2 = dict(nx=24, ny=24, nnp=12, nu=40, dx=1.0, dy=1.0, du=1.2, lsd=300.0, lso=150.0)
    hx = dict(nx=20, ny=14, nnp=12, nu=48, dt=1.5, du=1.2, lsd=300.0, lso=150.0)
    c3 = dict(nx=12, ny=12, nz=10, nnp=8, nu=20, nv=16, dx=1.0, dy=1.0, dz=1.0, du=1.5, dv=1.5, lsd=300.0,
              lso=150.0)
    return [
        ("A_B0_operator", f2, True),
        ("A_B1_operator", f2, True),
        ("A_H0_operator", hx, True),
        ("A_Hl_operator", hx, True),
        ("A_SF_operator", f2, False),
        ("A_B1_3D_operator", c3, False),
    ]


def record(mod):
    out = []
    for cls, geo, offsets in cases():
        log = []
        mod.CDLL = lambda *a, **k: _Dll(log)
        n = geo["nnp"]
        ang = 2 * np.pi * np.arange(n) / n + 0.1
        dz = np.linspace(-2.0, 2.0, n)
        drho = np.linspace(3.0, -3.0, n)
        kw = dict(dz=dz, drho=drho) if offsets else {}
        if cls in ("A_H0_operator", "A_Hl_operator"):
            args = (geo["nx"], geo["ny"], n, geo["nu"], geo["dt"], geo["du"], geo["lsd"], geo["lso"], ang)
        elif cls == "A_B1_3D_operator":
            args = (geo["nx"], geo["ny"], geo["nz"], n, geo["nu"], geo["nv"], geo["dx"], geo["dy"], geo["dz"],
                    geo["du"], geo["dv"], geo["lsd"], geo["lso"], ang)
        else:
            args = (geo["nx"], geo["ny"], n, geo["nu"], geo["dx"], geo["dy"], geo["du"], geo["lsd"], geo["lso"], ang)
        op = getattr(mod, cls)(*args, **kw)
        x = np.arange(op.shape[1], dtype=np.float64)
        y = np.arange(op.shape[0], dtype=np.float64)
        init = dict(log[0])
        # the module converts angles/dz/drho with astype (copies): map them
        # back by value through the pointers it passed
        roles = {}
        ptrs = [a for a in init["args"] if not isinstance(a, (int, float))]
        for role, ref in zip(("angles", "dz", "drho"), (ang, dz, drho)):
            if not ptrs:
                break
            p = ptrs.pop(0)
            addr = ctypes.cast(p, ctypes.c_void_p).value
            got = np.ctypeslib.as_array(ctypes.cast(addr, ctypes.POINTER(ctypes.c_double)), shape=(n,))
            assert np.array_equal(got, ref), role
            roles[role] = (addr, addr + 8 * n)
        init["args"] = [_describe(a, roles) for a in init["args"]]
        log.clear()
        op.matvec(x)
        fwd = dict(log[0])
        fwd["args"] = _pointer_roles(fwd["args"], ("y", "x"))
        log.clear()
        op.rmatvec(y)
        bwd = dict(log[0])
        bwd["args"] = _pointer_roles(bwd["args"], ("y", "x"))
        arrays = {"angles": ang.tolist()}
        if offsets:
            arrays.update(dz=dz.tolist(), drho=drho.tolist())
        out.append({"class": cls, "geometry": geo, "offsets": offsets, "arrays": arrays,
                    "shape": list(op.shape), "init": init, "forward": fwd, "backward": bwd})
    return out


def _pointer_roles(args, names):
    """(proj pointer, vol pointer, handle) as the module passes them."""
    res = []
    it = iter(names)
    for a in args:
        if isinstance(a, int) and a == 0xC0FFEE:
            res.append({"handle": True})
        elif isinstance(a, (int, float)):
            res.append(a)
        else:
            res.append({"array": next(it)})
    return res


def main(ref_root):
    mod = load_reference_module(ref_root)
    calls = record(mod)
    with open(OUT, "w") as f:
        json.dump({"source": "python/operators/operators.py of the reference, run unmodified",
                   "operators": calls}, f, indent=1)
    print(f"wrote {OUT}: {len(calls)} operators")


def default_reference():
    return os.environ.get("SGD_REFERENCE",
                          os.path.normpath(os.path.join(HERE, "..", "..", "..", "reference")))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else default_reference())
