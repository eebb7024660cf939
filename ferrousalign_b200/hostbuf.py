"""Reusable host output buffers for repeated calls of one kind (collection, CIGAR
regeneration, mate-rescue collection): each named buffer grows on demand and keeps its
storage, page-locked when `pinned`, so the library's device-to-host copies run at full bus
speed into pages that are already mapped instead of faulting fresh pages in every call.
Results built on them are views, valid until the next call that uses the same buffers."""
from __future__ import annotations

import numpy as np


class HostBuffers:
    def __init__(self, pinned: bool = True):
        self.pinned = pinned
        self._bufs: dict[str, np.ndarray] = {}

    def get(self, name: str, n: int, dtype) -> np.ndarray:
        """An array of n elements of dtype under `name`, reusing its storage when it fits."""
        dtype = np.dtype(dtype)
        nbytes = max(n, 1) * dtype.itemsize
        cur = self._bufs.get(name)
        if cur is None or cur.nbytes < nbytes:
            grown = nbytes + nbytes // 4
            if self.pinned:
                import torch
                cur = torch.empty(grown, dtype=torch.uint8).pin_memory().numpy()
            else:
                cur = np.empty(grown, np.uint8)
            self._bufs[name] = cur
        return cur[:nbytes].view(dtype)[:n]

    def capacity(self, name: str, dtype) -> int:
        """Elements of dtype the storage under `name` holds now (0 when there is none)."""
        cur = self._bufs.get(name)
        return 0 if cur is None else cur.nbytes // np.dtype(dtype).itemsize


def capacity(bufs: HostBuffers | None, name: str, dtype) -> int:
    """Elements of dtype `bufs`' buffer `name` holds now (0 without one)."""
    return bufs.capacity(name, dtype) if bufs is not None else 0


def out_array(bufs: HostBuffers | None, name: str, n: int, dtype, zero: bool = False) -> np.ndarray:
    """`bufs`' buffer `name`, or a fresh array (zeroed when `zero`) without buffers."""
    if bufs is not None:
        return bufs.get(name, n, dtype)
    return np.zeros(n, dtype) if zero else np.empty(n, dtype)
