"""Host logic of checkpoint / resume (augurv2_b200.checkpoint) on a CPU-only
stand-in sampler: what is saved, in-place restore, and the refusals."""
import pytest
import torch

from augurv2_b200.checkpoint import Checkpointable


class _Inner(Checkpointable):
    _ckpt_tensors = ("w",)
    _ckpt_scalars = ("steps",)

    def __init__(self):
        self.w = torch.zeros(3)
        self.steps = 0


class _Sampler(Checkpointable):
    _ckpt_tensors = ("x", "inner.w")
    _ckpt_scalars = ("iteration", "inner.steps")

    def __init__(self, n=4):
        self.x = torch.zeros(n, dtype=torch.float64)
        self.inner = _Inner()
        self.iteration = 0
        self.reloaded = 0

    def _ckpt_extra(self):
        return {"gen": 7}

    def _ckpt_load_extra(self, extra):
        self.extra = extra

    def _ckpt_after_load(self):
        self.reloaded += 1

    def step(self):
        self.x += torch.arange(self.x.numel(), dtype=torch.float64)
        self.inner.w += 1.0
        self.inner.steps += 1
        self.iteration += 1


def test_round_trip_restores_in_place(tmp_path):
    a = _Sampler()
    for _ in range(3):
        a.step()
    a.save(str(tmp_path / "c.pt"))
    b = _Sampler()
    ptr = b.x.data_ptr()
    b.load(str(tmp_path / "c.pt"))
    assert b.x.data_ptr() == ptr                    # copied into the existing storage
    assert torch.equal(a.x, b.x) and torch.equal(a.inner.w, b.inner.w)
    assert (b.iteration, b.inner.steps, b.reloaded, b.extra) == (3, 3, 1, {"gen": 7})
    a.step(); b.step()
    assert torch.equal(a.x, b.x)


def test_state_is_a_copy():
    a = _Sampler()
    d = a.state_dict()
    a.step()
    assert float(d["tensors"]["x"].sum()) == 0.0


def test_refuses_other_kind_and_other_shape():
    d = _Sampler().state_dict()
    with pytest.raises(ValueError):
        _Inner().load_state_dict(d)
    with pytest.raises(ValueError):
        _Sampler(n=5).load_state_dict(d)
