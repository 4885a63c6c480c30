"""Batching helpers and the device workspace pool.

``get_section_sizes`` / ``get_batches`` follow
``src/qttools/utils/mpi_utils.py:16-67`` and
``src/qttools/utils/solvers_utils.py:7-32`` so that energy batches are cut
exactly as in the reference solvers.
"""

from __future__ import annotations

import numpy as np
import torch


def get_section_sizes(num_elements: int, num_sections: int, strategy: str = "balanced"):
    quotient, remainder = divmod(num_elements, num_sections)
    if strategy == "balanced":
        sizes = remainder * [quotient + 1] + (num_sections - remainder) * [quotient]
    elif strategy == "greedy":
        sizes = [0] * num_sections
        for i in range(num_sections):
            sizes[i] = min(quotient + min(remainder, 1), num_elements - sum(sizes))
    else:
        raise ValueError(f"Invalid strategy: {strategy}")
    return sizes, max(sizes) * num_sections


def get_batches(num_sections: int, max_batch_size: int):
    sizes, _ = get_section_sizes(num_elements=num_sections,
                                 num_sections=num_sections // min(max_batch_size, num_sections))
    slices = np.hstack(([0], np.cumsum(np.array(sizes))))
    return sizes, slices


class WorkspacePool:
    """One growing device scratch buffer per (device, tag); reused across
    calls on the same stream."""

    def __init__(self):
        self._bufs: dict = {}

    def get(self, nbytes: int, device: torch.device, tag: str = "default") -> torch.Tensor:
        key = (device, tag)
        buf = self._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            self._bufs.pop(key, None)
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            self._bufs[key] = buf
        return buf

    def clear(self) -> None:
        self._bufs.clear()


workspace_pool = WorkspacePool()
