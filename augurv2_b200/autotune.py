"""Autotuner for the launch shapes of the batched tensor-core HLR pass.

The pass (ab_hlrb_logp_grad_cfg, csrc/hlrb.cu) has three knobs
(ab_hlrb_config): the forward GEMM's epilogue warps (4 or 8), the backward
GEMM's tile width (32, 64 or 128 gradient columns) and its number of row
splits.  Which shape is fastest depends on N, D, the number of chains and
the GPU: narrow D favours narrow backward tiles and many splits; small N
leaves too few forward tiles for eight epilogue warps to pay.  The tuner
times every candidate shape on the device with CUDA events (after warm-up,
median of a few passes) and keeps the fastest, caching the choice per
(GPU, N, D, C, pass kind) in a JSON file so later runs skip the timing.

The reference has no counterpart: its gradient is a thrust reduction per
component (compiler/augur/src/Low/SplitBlk.hs:382-389) with no tiling.
"""
import ctypes as C
import json
import os
import threading

from . import _native as N

DEFAULT_CACHE = os.environ.get(
    "AUGUR_B200_TUNE_CACHE",
    os.path.join(os.path.expanduser("~"), ".cache", "augurv2_b200", "autotune.json"))

FWD_WARPS = (4, 8, 16)
FWD_BN = (128, 256)
BWD_BN = (32, 64, 128)
BM, BK = 128, 64


class HlrbConfigC(C.Structure):
    _fields_ = [("fwd_warps", C.c_int), ("bwd_bn", C.c_int), ("bwd_splits", C.c_int), ("fwd_bn", C.c_int)]

    def as_dict(self):
        return {"fwd_warps": self.fwd_warps, "bwd_bn": self.bwd_bn, "bwd_splits": self.bwd_splits,
                "fwd_bn": self.fwd_bn}

    @classmethod
    def of(cls, d):
        return cls(int(d.get("fwd_warps", 0)), int(d.get("bwd_bn", 0)), int(d.get("bwd_splits", 0)),
                   int(d.get("fwd_bn", 0)))


def _ceil(a, b):
    return (a + b - 1) // b


def default_splits(N_, D, C_, bn, sms):
    """The library's built-in split count for a backward tile width (the
    same arithmetic as csrc/hlrb.cu: SMs / tiles, whole K steps per split)."""
    tiles = _ceil(C_, BM) * _ceil(D, bn)
    kb = _ceil(N_, 64) * 64 // BK
    sp = max(1, min(kb, sms // tiles))
    per = _ceil(kb, sp)
    return _ceil(kb, per)


def hlrb_candidates(N_, D, C_, sms):
    """Launch shapes worth timing for one problem: every forward tile width
    and epilogue width (4 epilogue warps only with 128-row tiles), the
    backward tile widths that are not mostly padding, and for each the
    built-in split count, half of it and twice it."""
    kb = _ceil(N_, 64) * 64 // BK
    widest = max(32, _ceil(D, 32) * 32)
    out = []
    for fbn in FWD_BN:
        for fw in FWD_WARPS:
            if fw == 4 and fbn == 256:
                continue
            for bn in BWD_BN:
                if bn > 2 * widest and bn != 32:
                    continue
                sp0 = default_splits(N_, D, C_, bn, sms)
                for sp in sorted({max(1, sp0 // 2), sp0, min(kb, 2 * sp0)}):
                    out.append({"fwd_warps": fw, "bwd_bn": bn, "bwd_splits": sp, "fwd_bn": fbn})
    return out


def select_best(candidates, timer):
    """(best candidate, {index: seconds}) with timer(candidate) -> seconds;
    ties go to the earlier candidate."""
    times = {}
    best, best_t = None, float("inf")
    for i, c in enumerate(candidates):
        t = float(timer(c))
        times[i] = t
        if t < best_t:
            best, best_t = c, t
    return best, times


class Autotuner:
    """Times candidate launch shapes and remembers the fastest per key."""

    def __init__(self, cache_path=DEFAULT_CACHE, reps=5, warmup=2, persist=True):
        self.cache_path = cache_path
        self.reps, self.warmup, self.persist = int(reps), int(warmup), bool(persist)
        self._lock = threading.Lock()
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            try:
                with open(cache_path) as f:
                    self.cache = json.load(f)
            except (OSError, ValueError):
                self.cache = {}
        self.timed = 0          # candidate timings run by this tuner

    def _save(self):
        if not (self.persist and self.cache_path):
            return
        d = os.path.dirname(self.cache_path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = self.cache_path + ".%d.tmp" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def lookup_or_tune(self, key, candidates, timer):
        with self._lock:
            if key in self.cache:
                return dict(self.cache[key]["config"])
        best, times = select_best(candidates, timer)
        self.timed += len(candidates)
        with self._lock:
            self.cache[key] = {"config": best, "seconds": times[candidates.index(best)],
                               "candidates": len(candidates)}
            self._save()
        return dict(best)

    def hlrb(self, data, C_, grad=True):
        """Fastest ab_hlrb_config (as a dict) for `data` (hlrb.HlrbData) with
        C_ chains; grad=False tunes the log-density-only pass."""
        import torch
        dev = data.device
        props = torch.cuda.get_device_properties(dev)
        key = "%s|hlrb|N=%d|D=%d|C=%d|%s" % (props.name, data.N, data.D, C_, "grad" if grad else "logp")
        cands = hlrb_candidates(data.N, data.D, C_, props.multi_processor_count)
        g = torch.Generator(device=dev)
        g.manual_seed(1234)
        theta = 0.1 * torch.randn((C_, data.D), generator=g, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)

        def timer(cand):
            cfg = HlrbConfigC.of(cand)
            work = data.workspace(C_, cfg)
            for _ in range(self.warmup):
                data.logp_grad(theta, grad, work=work, err=err, config=cfg)
            evs = []
            for _ in range(self.reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                data.logp_grad(theta, grad, work=work, err=err, config=cfg)
                b.record()
                evs.append((a, b))
            torch.cuda.synchronize()
            if int(err.item()) != 0:
                raise N.AugurError("device wait timed out while tuning %s" % cand)
            ts = sorted(a.elapsed_time(b) for a, b in evs)
            return ts[len(ts) // 2] / 1e3

        return self.lookup_or_tune(key, cands, timer)


_default = None


def default_tuner():
    global _default
    if _default is None:
        _default = Autotuner()
    return _default
