"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
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
