"""NVTX ranges around the samplers' phases (one range per call of a
sweep / run method), visible in Nsight Systems or ncu's NVTX filters.  The
reference has no tracing beyond log prints (pyaugur/augurlib.py:51-52).
Ranges are pushed only when AUGUR_B200_NVTX=1, so the default path pays
nothing."""
import contextlib
import functools
import os

_ON = os.environ.get("AUGUR_B200_NVTX", "0") == "1"


@contextlib.contextmanager
def nvtx_range(name):
    if not _ON:
        yield
        return
    import torch
    torch.cuda.nvtx.range_push(name)
    try:
        yield
    finally:
        torch.cuda.nvtx.range_pop()


def traced(name):
    """Decorator: run the method inside an NVTX range `name`."""
    def wrap(fn):
        @functools.wraps(fn)
        def inner(*a, **k):
            with nvtx_range(name):
                return fn(*a, **k)
        return inner
    return wrap
