"""Observables of the solved Green's functions.

``density`` follows ``src/quatrex/core/observables.py:8-31`` (no overlap,
one stack rank): the imaginary part of the diagonal of X^<. For a
``DSDBSparse`` it reads the container's diagonal; the fused device path
(:class:`quatrex_b200.EnergyPointSolver`) writes it directly from the
anti-Hermitian projection of the diagonal blocks.
"""

from __future__ import annotations

import numpy as np
import torch


def density(x, overlap=None):
    """Im diag(X) per orbital, shape ``(*stack_shape, N_orbitals)``."""
    if overlap is not None:
        raise NotImplementedError("the overlap-matrix density is not part of this path")
    d = x.diagonal()
    if isinstance(d, torch.Tensor):
        return d.imag
    return np.asarray(d).imag if isinstance(d, np.ndarray) else d.imag
