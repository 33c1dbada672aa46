"""Helpers shared by the GPU tests."""
from __future__ import annotations

import numpy as np
import torch


def dev64(a: np.ndarray) -> torch.Tensor:
    """uint64/int64 numpy -> CUDA int64 tensor (same bits)."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a.astype(np.int64, copy=False)).cuda()


def dev32(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32)).cuda()


def host_u64(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


def host_i64(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.int64)


# Tunings that force the ruling-set path (chase, recursion, propagation) even
# at small sizes, besides the default.
DEEP = dict(base_case_size=32, ruler_spacing=4, ruler_spacing_deep=3, max_levels=10)
SPARSE = dict(base_case_size=16, ruler_spacing=200, ruler_spacing_deep=50, max_levels=10)
