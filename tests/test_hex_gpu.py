"""Hexagonal-lattice projectors H0 and Hl on the GPU: parity with the FP64
oracle replica and with the reference library, adjoint tests."""
import numpy as np
import pytest

from geometry_cases import hex_case, rel_l2
from sgd_b200.phantom import hex_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# The hex kernels reproduce the reference's FP32 geometry (and its FP32 bin
# stepping), so against the FP64 replica they sit where the reference sits;
# the parity bar is the reference library itself.
TOL_ORACLE = 5e-5
TOL_PHANTOM = 1e-5
TOL_ADJOINT = 1e-6

# mode: (operator, keyword arguments, oracle mode, reference prefix, row pitch in dt)
MODES = {
    "h0": ("A_H0_operator", {}, "h0", "h0", 1.5),
    "h0c": ("A_H0_operator", {"exact_bounds": True}, "h0c", None, 1.5),
    "hl": ("A_Hl_operator", {}, "hl", "hl", 0.5),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def make(mode, case):
    import sgd_b200.operators as ops
    nl, nc, nu, dt, du, lsd, lso, ang = hex_case(case)
    cls, kw = MODES[mode][0], MODES[mode][1]
    A = getattr(ops, cls)(nl, nc, len(ang), nu, dt, du, lsd, lso, ang, **kw)
    x = hex_phantom(nl, nc, dt, MODES[mode][4] * dt, seed=0).ravel()
    return A, (nl, nc, nu, dt, du, lsd, lso, ang), x


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("case", ["small", "tall"])
def test_matches_fp64_oracle(oracle_mod, mode, case):
    A, g, x = make(mode, case)
    om = MODES[mode][2]
    b_ref, cnt = oracle_mod.hex_forward(om, x, *g)
    assert rel_l2(A.matvec(x), b_ref) < TOL_ORACLE
    assert rel_l2(A.rmatvec(b_ref), oracle_mod.hex_backward(om, b_ref, *g)) < TOL_ORACLE
    assert abs(A.conv_count - cnt) <= 1e-4 * cnt + 3


@pytest.mark.parametrize("mode", ["h0", "hl"])
@pytest.mark.parametrize("case", ["small", "2e18"])
def test_matches_reference_library(mode, case):
    import reflib
    if not reflib.available():
        pytest.fail("reference library oracle/_ref/libnetwork.so not built (make -C oracle ref)")
    A, g, x = make(mode, case if case == "small" else f"{mode}_{case}")
    R = reflib.RefHex(MODES[mode][3], *g)
    b_ref, cnt = R.forward(x)
    assert rel_l2(A.matvec(x), b_ref) < TOL_PHANTOM
    assert rel_l2(A.rmatvec(b_ref), R.backward(b_ref)) < TOL_PHANTOM
    assert abs(A.conv_count - cnt) <= 1e-4 * cnt + 3


@pytest.mark.parametrize("mode", ["h0c", "hl"])
@pytest.mark.parametrize("case", ["small", "2e18"])
def test_adjoint_dot_product(mode, case):
    A, g, _ = make(mode, case if case == "small" else ("h0" if mode == "h0c" else "hl") + "_" + case)
    rng = np.random.default_rng(1234)
    x = rng.standard_normal(A.shape[1])
    nl, nc = g[0], g[1]
    x.reshape(nc, nl)[nc - 1, 1::2] = 0.0  # not sites
    y = rng.standard_normal(A.shape[0])
    lhs = float(np.dot(A.matvec(x), y))
    rhs = float(np.dot(x, A.rmatvec(y)))
    assert abs(lhs - rhs) / abs(lhs) < TOL_ADJOINT


def test_h0_reference_mode_loses_mass_the_corrected_mode_keeps(oracle_mod):
    """The reference's H0 bounds use the 0.5 dt row pitch of its projection
    matrices (layers/A_H0.cu:556) for sites placed at 1.5 dt: the projection of
    a constant image loses most of its mass; the corrected bounds keep it."""
    Ar, g, _ = make("h0", "small")
    Ac, _, _ = make("h0c", "small")
    nl, nc = g[0], g[1]
    ones = hex_phantom(nl, nc, g[3], 1.5 * g[3], seed=0).ravel() * 0 + 1.0
    ones.reshape(nc, nl)[nc - 1, 1::2] = 0.0
    sr, sc = Ar.matvec(ones).sum(), Ac.matvec(ones).sum()
    assert sc > 2.0 * sr


def test_h0_corrected_against_exact_hexagon_projection(oracle_mod):
    """The GPU H0 with the true hexagon bounds against the exact FP64
    bin-averaged chords of the hexagon indicator (three times, the H0 basis's
    normalisation): the model error of the footprint formula."""
    from sgd_b200.operators import A_H0_operator
    nl, nc, nu, dt, du, lsd, lso = 16, 12, 60, 2.0, 1.5, 1085.6, 595.0
    ang = np.array([0.3, 1.1, np.pi / 4, 2.5])
    M = oracle_mod.exact_hex_matrix(nl, nc, nu, dt, du, lsd, lso, ang)
    A = A_H0_operator(nl, nc, len(ang), nu, dt, du, lsd, lso, ang, exact_bounds=True)
    x = np.random.default_rng(0).random(nc * nl)
    odd_last = [(nc - 1) * nl + il for il in range(1, nl, 2)]
    x[odd_last] = 0.0  # absent sites of the odd rows
    assert rel_l2(A.matvec(x), 3.0 * (M @ x)) < 1e-4


def test_hl_against_exact_linear_element_projection(oracle_mod):
    """The GPU Hl against the exact FP64 bin-averaged line integrals of the
    Courant hat on the lattice (its FP64 formula sits 7.5e-6 from them)."""
    from sgd_b200.operators import A_Hl_operator
    nl, nc, nu, dt, du, lsd, lso = 24, 12, 60, 2.0, 1.5, 1085.6, 595.0
    ang = np.array([0.3, 1.1, np.pi / 4, 2.5])
    M = oracle_mod.exact_hl_matrix(nl, nc, nu, dt, du, lsd, lso, ang)
    A = A_Hl_operator(nl, nc, len(ang), nu, dt, du, lsd, lso, ang)
    x = np.random.default_rng(0).random(nc * nl)
    x[[(nc - 1) * nl + il for il in range(1, nl, 2)]] = 0.0  # absent sites of the odd rows
    assert rel_l2(A.matvec(x), M @ x) < 2e-4
