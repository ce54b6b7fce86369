"""Checkpoint and resume of sampler state.

The reference keeps no checkpoints (its runtime state lives in process
globals, cbits/augur_mcmclib.h:44-45).  Here every sampler's state is a set
of device tensors plus a few host scalars, and every random draw is
addressed by (seed, element, iteration, tag) in a counter-based Philox
stream, so the state below is all a chain needs: a sampler restored from a
checkpoint continues bit for bit as the uninterrupted run would.

A sampler class lists its state in `_ckpt_tensors` (attribute paths of
torch tensors, copied back in place so captured CUDA graphs and the C
descriptors that hold their addresses stay valid) and `_ckpt_scalars` (host
values), and may add `_ckpt_extra` / `_ckpt_load_extra` for anything else
and `_ckpt_after_load` to re-derive device state.
"""
import torch


def _get(obj, path):
    for p in path.split("."):
        obj = getattr(obj, p)
    return obj


def _set(obj, path, value):
    head, _, last = path.rpartition(".")
    if head:
        obj = _get(obj, head)
    setattr(obj, last, value)


class Checkpointable:
    _ckpt_tensors = ()
    _ckpt_scalars = ()

    def _ckpt_extra(self):
        return None

    def _ckpt_load_extra(self, extra):
        pass

    def _ckpt_after_load(self):
        pass

    def state_dict(self):
        """Host copy of the sampler's state (torch.save-able)."""
        if torch.cuda.is_available():
            torch.cuda.synchronize()
        return {"kind": type(self).__name__,
                "tensors": {n: _get(self, n).detach().to("cpu", copy=True) for n in self._ckpt_tensors},
                "scalars": {n: _get(self, n) for n in self._ckpt_scalars},
                "extra": self._ckpt_extra()}

    def load_state_dict(self, d):
        """Restore a state_dict() of a sampler built with the same sizes."""
        if d.get("kind") != type(self).__name__:
            raise ValueError("checkpoint of a %s, not a %s" % (d.get("kind"), type(self).__name__))
        for n in self._ckpt_tensors:
            src, dst = d["tensors"][n], _get(self, n)
            if tuple(src.shape) != tuple(dst.shape) or src.dtype != dst.dtype:
                raise ValueError("checkpoint tensor %s is %s %s, the sampler has %s %s"
                                 % (n, tuple(src.shape), src.dtype, tuple(dst.shape), dst.dtype))
            dst.copy_(src)
        for n in self._ckpt_scalars:
            _set(self, n, d["scalars"][n])
        self._ckpt_load_extra(d.get("extra"))
        self._ckpt_after_load()
        if torch.cuda.is_available():
            torch.cuda.synchronize()

    def save(self, path):
        torch.save(self.state_dict(), path)

    def load(self, path):
        self.load_state_dict(torch.load(path, weights_only=False))
