"""Checkpoint and resume of the warm-start network's training, on the CPU.

The network's state (FP32 master weights, biases, Adam moments and step)
round-trips through a file on host tensors; train() interrupted after an
epoch and started again on the same checkpoint continues exactly as the
uninterrupted run (same batches, same step sizes, same losses).  No kernel
runs: the network is built on the CPU device, and the resume test trains a
stand-in network that records what it is given."""
import os
import sys

import pytest

torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _cpu_net(seed=0, channels=(1, 8, 8, 1)):
    from sgd_b200.cnn import WarmStartCNN
    return WarmStartCNN(channels=channels, seed=seed, device=torch.device("cpu"))


def test_network_state_round_trips_through_a_file(tmp_path):
    a = _cpu_net(seed=1)
    for k, p in enumerate(a.params):  # a trained-looking state: non-zero moments
        p.add_(0.25 * (k + 1))
        a.m[k].fill_(0.5 + k)
        a.v[k].fill_(2.0 + k)
    a.step_count = 17
    a.save(str(tmp_path / "net.pt"))
    b = _cpu_net(seed=2)
    b.load(str(tmp_path / "net.pt"))
    for key in ("w32", "b", "m", "v"):
        for pa, pb in zip(getattr(a, key), getattr(b, key)):
            assert torch.equal(pa, pb)
    for w16, w32 in zip(b.w16, b.w32):  # the BF16 copies follow the masters
        assert w16.dtype == torch.bfloat16 and torch.equal(w16, w32.to(torch.bfloat16))
    assert b.step_count == 17


def test_network_state_rejects_another_architecture():
    a = _cpu_net(channels=(1, 8, 8, 1))
    with pytest.raises(ValueError, match="channels"):
        _cpu_net(channels=(1, 4, 4, 1)).load_state_dict(a.state_dict())
    sd = a.state_dict()
    sd["m"] = sd["m"][:-1]
    with pytest.raises(ValueError, match="shapes"):
        a.load_state_dict(sd)


class _Interrupted(Exception):
    pass


class _RecordingNet:
    """Stand-in for WarmStartCNN: records each batch's sample indices and step
    size; its state is the number of steps taken."""

    def __init__(self, fail_at=None):
        self.calls, self.steps, self.fail_at = [], 0, fail_at

    def train_step(self, x, t, lr):
        if self.fail_at is not None and self.steps == self.fail_at:
            raise _Interrupted()
        self.steps += 1
        ids = x[:, 0, 0, 0].long().tolist()
        self.calls.append((ids, lr))
        return torch.tensor([float(sum(ids))], dtype=torch.float64)

    def state_dict(self):
        return {"steps": self.steps}

    def load_state_dict(self, sd):
        self.steps = int(sd["steps"])


def test_training_resumes_where_it_stopped(tmp_path):
    from sgd_b200.asd import train
    n, batch, epochs = 24, 4, 5
    x = torch.arange(n, dtype=torch.float32).reshape(n, 1, 1).expand(n, 2, 2).contiguous()
    t = torch.zeros_like(x)
    kw = dict(epochs=epochs, batch=batch, lr=1e-3, lr_final=1e-4, seed=3)

    full = _RecordingNet()
    losses_full = train(full, x, t, **kw)
    per_epoch = n // batch

    ck = str(tmp_path / "train.ck")
    first = _RecordingNet(fail_at=2 * per_epoch + 1)  # dies inside the third epoch
    with pytest.raises(_Interrupted):
        train(first, x, t, checkpoint=ck, **kw)
    assert first.calls == full.calls[:2 * per_epoch + 1]

    second = _RecordingNet()
    losses = train(second, x, t, checkpoint=ck, **kw)
    assert second.steps == full.steps  # restored from the checkpoint, then continued
    assert second.calls == full.calls[2 * per_epoch:]  # the third epoch is redone from its start
    assert losses == losses_full

    with pytest.raises(ValueError, match="another training run"):
        train(_RecordingNet(), x, t, checkpoint=ck, **dict(kw, seed=4))
