"""The CUDA device every buffer lives on (one process per GPU)."""

from __future__ import annotations

import os

_DEV = None


def device():
    """``cuda:<LOCAL_RANK>``; raises when no GPU is visible (no CPU fallback)."""
    global _DEV
    if _DEV is None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("jaxrens_b200 needs a CUDA device; none is visible")
        _DEV = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    return _DEV
