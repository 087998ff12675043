"""Batched B1 projection (persistent launches, CUDA graph, autotuner) against
the per-slice projector and against the FP64 oracle."""
import numpy as np
import pytest

from geometry_cases import LSD, LSO, rel_l2
from sgd_b200.phantom import ellipse_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def mixed_slices():
    """Uneven sizes, views and bin counts, a snapped 45-degree view, nx != ny."""
    return [
        (64, 64, 92, 1.0, 1.0, 1.0, LSD, LSO, 2 * np.pi * np.arange(24) / 24),
        (96, 80, 140, 0.8, 0.9, 1.0, LSD, LSO, np.array([0.1, np.pi / 4, 1.9, 3.3, 5.0])),
        (48, 48, 70, 1.5, 1.5, 1.2, 900.0, 500.0, 2 * np.pi * np.arange(36) / 36),
        (128, 128, 185, 0.5, 0.5, 1.0, LSD, LSO, 2 * np.pi * np.arange(60) / 60),
    ]


def per_slice(slices, imgs, sinos):
    """Per-slice single-layer projectors on the same device inputs."""
    from sgd_b200.torch_ops import FanProjector
    fw, bw = [], []
    for s, x, y in zip(slices, imgs, sinos):
        P = FanProjector("b1", s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], s[8])
        fw.append(P.forward(x.contiguous()))
        bw.append(P.backward(y.contiguous()))
    return fw, bw


def fill(batch, seed=0):
    img = batch.image_arena()
    for k, v in enumerate(batch.images(img)):
        s = batch.slices[k]
        v.copy_(torch.tensor(ellipse_phantom(s[0], s[1], s[3], s[4], seed=seed + k), dtype=torch.float32))
    sino = batch.sinogram_arena()
    sino.copy_(torch.rand(sino.numel(), generator=torch.Generator().manual_seed(seed)).cuda())
    return img, sino


@pytest.mark.parametrize("vc", [2, 4, 8])
def test_batch_slices_match_fp64_oracle(oracle_mod, vc):
    """Every slice of an uneven batch, forward and back, against the FP64
    replica of the reference formula (layers/A_B1.cu:62-353) at the
    projector tests' parity bar."""
    from sgd_b200.batch import B1Batch
    slices = mixed_slices()
    B = B1Batch(slices)
    B.set_variant(4, vc)
    img, sino = fill(B, seed=11)
    out_s = B.forward(img)
    out_i = B.backward(sino)
    torch.cuda.synchronize()
    B.status()
    for k, s in enumerate(slices):
        nx, ny, nu, dx, dy, du, lsd, lso, ang = s
        x = B.images(img)[k].double().cpu().numpy().ravel()
        y = B.sinograms(sino)[k].double().cpu().numpy().ravel()
        b_ref, _ = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
        xt_ref = oracle_mod.b1_backward(y, nx, ny, nu, dx, dy, du, lsd, lso, ang)
        assert rel_l2(B.sinograms(out_s)[k].double().cpu().numpy().ravel(), b_ref) < 1e-5, k
        assert rel_l2(B.images(out_i)[k].double().cpu().numpy().ravel(), xt_ref) < 1e-5, k


def test_batch_equals_per_slice_projector_bitwise():
    from sgd_b200.batch import B1Batch
    slices = mixed_slices()
    B = B1Batch(slices)
    B.set_variant(8, 4)  # the single-slice kernels' shape
    img, sino = fill(B)
    out_s = B.forward(img)
    out_i = B.backward(sino)
    torch.cuda.synchronize()
    B.status()
    fw, bw = per_slice(slices, B.images(img), B.sinograms(sino))
    for a, b in zip(B.sinograms(out_s), fw):
        assert torch.equal(a, b)
    for a, b in zip(B.images(out_i), bw):
        assert torch.equal(a, b)


@pytest.mark.parametrize("fw", [4, 8, 16])
@pytest.mark.parametrize("vc", [2, 4, 8])
def test_every_variant_matches(fw, vc):
    from sgd_b200.batch import B1Batch
    slices = mixed_slices()
    B = B1Batch(slices)
    B.set_variant(fw, vc)
    img, sino = fill(B, seed=3)
    out_s = B.forward(img)
    out_i = B.backward(sino)
    torch.cuda.synchronize()
    B.status()
    fw_ref, bw_ref = per_slice(slices, B.images(img), B.sinograms(sino))
    for a, b in zip(B.sinograms(out_s), fw_ref):
        assert torch.equal(a, b)  # one warp per row whatever the item size
    for a, b in zip(B.images(out_i), bw_ref):
        assert rel_l2(a.double().cpu().numpy(), b.double().cpu().numpy()) < 1e-6


def test_graph_replay_matches_direct_launch():
    from sgd_b200.batch import B1Batch
    B = B1Batch(mixed_slices())
    img, sino = fill(B, seed=5)
    out_s, out_i = B.sinogram_arena(), B.image_arena()
    B.capture(img, out_s, sino, out_i)
    for _ in range(3):
        B.replay()
    torch.cuda.synchronize()
    B.status()
    ref_s = B.forward(img)
    ref_i = B.backward(sino)
    torch.cuda.synchronize()
    assert torch.equal(out_s, ref_s)
    assert torch.equal(out_i, ref_i)
    # new inputs in the same arenas are picked up by the next replay
    img.mul_(2.0)
    B.replay()
    torch.cuda.synchronize()
    assert rel_l2(out_s.double().cpu().numpy(), 2 * ref_s.double().cpu().numpy()) < 1e-6


def test_autotuner_measures_then_loads_from_cache(tmp_path):
    from sgd_b200.batch import B1Batch
    cache = str(tmp_path / "tune.txt")
    B = B1Batch(mixed_slices())
    fw, vc, loaded = B.tune(cache)
    assert not loaded and fw in (4, 8, 16) and vc in (2, 4, 8)
    C = B1Batch(mixed_slices())
    fw2, vc2, loaded2 = C.tune(cache)
    assert loaded2 and (fw2, vc2) == (fw, vc)
    with open(cache) as f:
        assert len(f.read().splitlines()) == 1
    img, sino = fill(C, seed=7)
    out = C.backward(sino)
    torch.cuda.synchronize()
    C.status()
    assert torch.isfinite(out).all()


def test_identical_slices_share_tables_and_stay_independent():
    from sgd_b200.batch import B1Batch
    s = mixed_slices()[0]
    B = B1Batch([s, s, s])
    img, sino = fill(B, seed=9)
    out = B.forward(img)
    torch.cuda.synchronize()
    fw, _ = per_slice([s] * 3, B.images(img), B.sinograms(sino))
    for a, b in zip(B.sinograms(out), fw):
        assert torch.equal(a, b)


def test_uneven_48_slice_batch_matches_per_slice():
    """The 48-slice uneven workload (sides 256/384/512, 360/540/720 views)."""
    from sgd_b200.batch import B1Batch, uneven_slices
    slices = uneven_slices(seed=0)
    B = B1Batch(slices)
    img, sino = fill(B, seed=11)
    out_s = B.forward(img)
    out_i = B.backward(sino)
    torch.cuda.synchronize()
    B.status()
    for k in (0, 17, 47):
        fw, bw = per_slice([slices[k]], [B.images(img)[k]], [B.sinograms(sino)[k]])
        assert torch.equal(B.sinograms(out_s)[k], fw[0])
        assert torch.equal(B.images(out_i)[k], bw[0])


def test_bad_variant_raises():
    from sgd_b200 import _lib
    from sgd_b200.batch import B1Batch
    B = B1Batch(mixed_slices()[:1])
    with pytest.raises(_lib.ProjectorError):
        B.set_variant(5, 4)
