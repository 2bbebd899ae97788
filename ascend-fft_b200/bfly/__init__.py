"""bfly: batched power-of-two fp32 FFTs on NVIDIA B200 (sm_100a).

A drop-in for the plan API of TruNcat3/ascend-fft (Context.init(profile, space, kernel),
select / make_plan, Plan.run / run_r2c / run_c2r / measure) plus asynchronous device-pointer
entry points and torch.fft-style functions with autograd.  All transforms run in the
hand-written CUDA kernels of libbfly_b200.so; importing the transforms without the built
library raises.
"""
from ._lib import LIB_PATH, load
from .core import (DEFAULT_CANDIDATE, DEFAULT_PROFILE, DEFAULT_SPACE, BflyError, Context, Plan)

__all__ = ["LIB_PATH", "load", "Context", "Plan", "BflyError", "DEFAULT_PROFILE", "DEFAULT_SPACE",
           "DEFAULT_CANDIDATE", "fft", "ifft", "fft2", "ifft2", "rfft", "irfft", "rfft2", "irfft2", "stft", "istft", "c2c", "c2c_axis",
           "c2c_2d", "r2c", "c2r", "c2c_tensor", "plan_for", "autotune"]


def __getattr__(name):
    # torch-level ops are imported lazily so the plan API works without importing torch.
    if name in ("fft", "ifft", "fft2", "ifft2", "rfft", "irfft", "rfft2", "irfft2", "stft", "istft", "c2c", "c2c_axis", "c2c_2d", "r2c", "c2r",
                "c2c_tensor", "plan_for", "autotune"):
        from . import ops
        return getattr(ops, name)
    raise AttributeError(name)
