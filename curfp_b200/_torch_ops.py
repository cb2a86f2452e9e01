"""Loader of the torch extension (curfp_b200/csrc_torch/torch_ops.cpp): the
RFP routines and their adjoints as torch operators, torch.ops.curfp_b200.*,
each run on torch's current CUDA stream.  Built in-tree by
``python -m curfp_b200.build``; there is no fallback."""
from __future__ import annotations

from pathlib import Path

import torch

EXT_PATH = Path(__file__).resolve().parent / "_torch_build" / "curfp_torch_ops.so"

_loaded = False


def ops():
    """torch.ops.curfp_b200, loading the extension on first use."""
    global _loaded
    if not _loaded:
        if not EXT_PATH.exists():
            raise ImportError(
                f"{EXT_PATH} is missing: build it with `python -m curfp_b200.build` "
                "(the torch extension is required; there is no fallback)")
        from . import _lib
        _lib.load()  # the C library the extension links (same in-tree copy)
        torch.ops.load_library(str(EXT_PATH))
        _loaded = True
    return torch.ops.curfp_b200
