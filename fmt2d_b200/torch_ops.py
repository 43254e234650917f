"""PyTorch operators of the hot path: torch.ops.fmt2d.{forward, field, trace,
frechet_rows, lsqr}, registered by the in-tree library
fmt2d_b200/_lib/libfmt2d_torch.so (built by fmt2d_b200.build) on the same C
ABI as the ctypes binding.  They take and return tensors (CUDA or CPU),
order the library's stream after the caller's current CUDA stream, and
return complete results.  A context is an api.Fmt2d; its C handle is passed
as an int."""
from __future__ import annotations

import os

import torch

from . import _native

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libfmt2d_torch.so")
OPS = ("forward", "field", "trace", "frechet_rows", "lsqr")
_loaded = False


def load():
    """Register torch.ops.fmt2d.* (once); raises if the library is missing."""
    global _loaded
    if _loaded:
        return torch.ops.fmt2d
    if not os.path.exists(LIB_PATH):
        raise _native.Fmt2dError(f"PyTorch operators not built: {LIB_PATH} "
                                 "(run fmt2d_b200.build.build())")
    _native.lib()                 # the C-ABI library the operators link against
    torch.ops.load_library(LIB_PATH)
    _loaded = True
    return torch.ops.fmt2d


def handle(g) -> int:
    """The C context handle of an api.Fmt2d, as the operators take it."""
    return int(g.h.value)
