"""Helpers shared by the tests: moving numpy arrays through torch device
buffers bit-for-bit, and reading 16-byte results."""
from __future__ import annotations

import numpy as np

RESULT_DTYPE = np.dtype([("found", np.uint8), ("pad", np.uint8, 7), ("value", np.uint64)])

_VIEW = {
    np.dtype(np.uint64): np.int64,
    np.dtype(np.uint32): np.int32,
    np.dtype(np.uint8): np.uint8,
    np.dtype(np.bool_): np.uint8,
}


def dev(a: np.ndarray):
    """numpy -> CUDA tensor with the same bytes (unsigned views as signed)."""
    import torch
    a = np.ascontiguousarray(a)
    v = a.view(_VIEW.get(a.dtype, a.dtype))
    return torch.from_numpy(v.copy()).cuda()


def host(t, dtype) -> np.ndarray:
    """CUDA tensor -> numpy array of `dtype` (same bytes)."""
    return t.cpu().numpy().view(dtype).reshape(-1)


def results_buf(n: int):
    import torch
    return torch.full((n, 2), -1, dtype=torch.int64, device="cuda")


def results(t) -> np.ndarray:
    return t.cpu().numpy().reshape(-1).view(RESULT_DTYPE)


def same_results(got: np.ndarray, want: np.ndarray) -> bool:
    """found bits equal everywhere; values equal everywhere (misses are 0 on
    both sides: the library writes 0, the oracle writes 0)."""
    return bool(np.array_equal(got["found"], want["found"]) and
                np.array_equal(got["value"], want["value"]))


def first_mismatch(got: np.ndarray, want: np.ndarray) -> str:
    bad = np.nonzero((got["found"] != want["found"]) | (got["value"] != want["value"]))[0]
    if len(bad) == 0:
        return "none"
    i = int(bad[0])
    return (f"{len(bad)} mismatches; first at {i}: got ({got['found'][i]}, {got['value'][i]:#x}) "
            f"want ({want['found'][i]}, {want['value'][i]:#x})")
