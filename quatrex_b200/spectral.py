"""Spectral open-boundary condition with Beyn's contour-integral NEVP solver.

``Beyn`` mirrors ``qttools.nevp.Beyn`` (``src/qttools/nevp/beyn.py:14-379``)
and ``Spectral`` mirrors ``qttools.boundary_conditions.obc.Spectral``
(``src/qttools/boundary_conditions/obc/spectral.py:15-629``), the OBC
algorithm quatrex selects by default (``src/quatrex/core/config.py:419``).
Same constructor arguments, same call signatures and return values.

Where the work runs:

* on the GPU (libqtx_b200): the 2 x ``num_quad_points`` operator inverses
  per energy and the two contour moments (``qtx_beyn_moments``), the
  projections q0 Y, q1 Y, the mode products a_x V, the rank-m product that
  forms x_ii a_ij, and every n x n inverse and refinement step of the
  surface Green's function;
* on the host (NumPy LAPACK), as in the reference's default compute
  location ``"numpy"``: the SVD (or QR) of the m_0-column projected moment,
  the eigenproblem of the reduced m x m system, and the per-mode masks.

Only ``block_sections = 1`` (the quatrex default) and the surface Green's
function output (``return_injected = False``, what the electron solver's
retarded boundary self-energy uses) are provided.
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from . import _native
from ._interop import default_device, from_device, mat
from .obc import OBCSolver, _dev3, _stream, fixed_point_refine, inverse
from .utils import workspace_pool

_C128 = torch.complex128
_NULL = _native.NULL_MAT


def _zgemm(a: torch.Tensor, b: torch.Tensor, out: torch.Tensor, addend: torch.Tensor | None = None,
           beta: float = 1.0) -> torch.Tensor:
    """out = a @ b (+ beta * addend) on the FP64 tensor cores, batched."""
    lib = _native.load()
    batch, m, k = a.shape
    n = b.shape[-1]
    _native.check(lib.qtx_zgemm_batched(m, n, k, batch, 1.0, 0.0, mat(a), 0, mat(b), 0, beta, 0.0,
                                        mat(addend) if addend is not None else _NULL, 0, mat(out),
                                        _stream(a.device)))
    return out


class Beyn:
    """Beyn's integral method for the lead's polynomial eigenvalue problem
    (``beyn.py:14-97``). The random subspace guess comes from
    ``numpy.random.default_rng(42)``, created with the instance and advanced
    by every call, as in the reference, so the same sequence of calls sees the
    same guesses. ``num_threads_contour``, ``eig_compute_location``,
    ``project_compute_location``, ``contour_batch_size`` and
    ``use_pinned_memory`` are accepted for interface compatibility; the
    contour runs on the GPU and the small dense problems on the host."""

    def __init__(self, r_o: float, r_i: float, m_0: int, num_quad_points: int, num_threads_contour: int = 1024,
                 eig_compute_location: str = "numpy", project_compute_location: str = "numpy",
                 use_qr: bool = False, contour_batch_size: int | None = None, use_pinned_memory: bool = True,
                 device: torch.device | None = None):
        self.r_o = r_o
        self.r_i = r_i
        self.m_0 = m_0
        self.num_quad_points = num_quad_points
        self.num_threads_contour = num_threads_contour
        self.eig_compute_location = eig_compute_location
        self.project_compute_location = project_compute_location
        self.use_qr = use_qr
        self.contour_batch_size = num_quad_points if contour_batch_size is None else contour_batch_size
        self.use_pinned_memory = use_pinned_memory
        self.device = device
        self.rng = np.random.default_rng(42)

    def moments(self, a_ji: torch.Tensor, a_ii: torch.Tensor, a_ij: torch.Tensor):
        """Contour moments q0, q1 of (B, d, d) device stacks (beyn.py:166-220)."""
        lib = _native.load()
        batch, d = a_ii.shape[0], a_ii.shape[-1]
        q0, q1 = torch.empty_like(a_ii), torch.empty_like(a_ii)
        ws = workspace_pool.get(lib.qtx_beyn_moments_workspace(d, batch, self.num_quad_points), a_ii.device,
                                "beyn")
        info = torch.zeros(batch, dtype=torch.int32, device=a_ii.device)
        _native.check(lib.qtx_beyn_moments(d, batch, mat(a_ji), mat(a_ii), mat(a_ij), float(self.r_o),
                                           float(self.r_i), int(self.num_quad_points), mat(q0), mat(q1),
                                           info.data_ptr(), ws.data_ptr(), ws.numel(), _stream(a_ii.device)))
        if bool((info != 0).any()):
            raise np.linalg.LinAlgError("Singular matrix")
        return q0, q1

    def _one_sided(self, a_ji, a_ii, a_ij):
        """beyn.py:282-326 (project, then solve the reduced system)."""
        batch, d = a_ii.shape[0], a_ii.shape[-1]
        y = self.rng.random((batch, d, self.m_0)) + 1j * self.rng.random((batch, d, self.m_0))
        q0, q1 = self.moments(a_ji, a_ii, a_ij)
        yd = torch.from_numpy(y).to(a_ii.device)
        p0 = _zgemm(q0, yd, torch.empty((batch, d, self.m_0), dtype=_C128, device=a_ii.device))
        p1 = _zgemm(q1, yd, torch.empty((batch, d, self.m_0), dtype=_C128, device=a_ii.device))
        p0, p1 = p0.cpu().numpy(), p1.cpu().numpy()
        ws = np.zeros((batch, self.m_0), dtype=np.complex128)
        vs = y.copy()
        for i in range(batch):
            if self.use_qr:  # _project_qr, beyn.py:146-164
                q, r = np.linalg.qr(p0[i])
                a = q.conj().T @ p1[i] @ np.linalg.inv(r)
                p_back = q
            else:  # _project_svd, beyn.py:99-145 (singular values in the input dtype)
                u, s, vh = np.linalg.svd(p0[i], full_matrices=False)
                s = s.astype(p0.dtype)
                keep = np.where(s > s.max() * d * np.finfo(p0.dtype).eps)[0]
                u, s, vh = u[:, keep], s[keep], vh[keep, :]
                a = u.conj().T @ p1[i] @ vh.conj().T / s
                p_back = u
            w, v = np.linalg.eig(a)  # _solve_reduced_system, beyn.py:223-280
            ws[i, :len(w)] = w
            vs[i, :, :len(w)] = p_back @ v
        return ws, vs

    def __call__(self, a_xx):
        """beyn.py:328-379: eigenvalues (..., m_0) and right eigenvectors
        (..., d, m_0) as NumPy arrays for the coefficient blocks a_xx from
        lowest to highest order (three blocks: a_ji, a_ii, a_ij)."""
        if len(a_xx) != 3:
            raise NotImplementedError("the contour kernel takes the three blocks of block_sections = 1")
        device = self.device or default_device()
        batch_shape = tuple(a_xx[0].shape[:-2])
        d = int(a_xx[0].shape[-1])
        if d < self.m_0 and self.use_qr:
            warnings.warn(f"Subspace guess {self.m_0} is larger than the dimension of the system {d}. "
                          f"Setting subspace guess to {d}.")
            old, self.m_0 = self.m_0, d
        else:
            old = None
        blocks = [_dev3(a, device) for a in a_xx]
        ws, vs = self._one_sided(*blocks)
        m0 = self.m_0
        if old is not None:
            self.m_0 = old
        return ws.reshape(*batch_shape, m0), vs.reshape(*batch_shape, d, m0)


class Spectral(OBCSolver):
    """Spectral OBC solver (``spectral.py:15-105``): the surface Green's
    function from the reflected eigenmodes of the lead found by ``nevp``."""

    def __init__(self, nevp: Beyn, block_sections: int = 1, min_decay: float = 1e-3, max_decay: float = 6.9,
                 num_ref_iterations: int = 2, min_propagation: float = 0.01, residual_tolerance: float = 1e-3,
                 residual_normalization: bool = True, warning_threshold: float = 1e-1, eta_decay: float = 1e-14,
                 device: torch.device | None = None) -> None:
        self.nevp = nevp
        self.min_decay = min_decay
        self.max_decay = max_decay
        self.num_ref_iterations = num_ref_iterations
        self.block_sections = block_sections
        self.min_propagation = min_propagation
        self.residual_tolerance = residual_tolerance
        self.residual_normalization = residual_normalization
        self.warning_threshold = warning_threshold
        self.eta_decay = eta_decay
        self.device = device
        if self.num_ref_iterations < 1:
            raise ValueError("Number of refinement iterations must be at least 1.")
        if self.block_sections != 1:
            raise NotImplementedError("only block_sections = 1 (the quatrex default) is provided")

    def _find_reflected_modes(self, ws, vs, prods):
        """spectral.py:197-304 (no injection) on host arrays; prods[x] are
        the device products a_x @ vs (x = a_ji, a_ii, a_ij) brought back."""
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            products = sum(p * ws[..., np.newaxis, :] ** (i - 1) for i, p in enumerate(prods))
            residuals = np.linalg.norm(products, axis=-2)
            residuals /= np.linalg.norm(vs, axis=-2)
            if self.residual_normalization:
                residuals /= np.abs(ws)
            # _compute_dE_dk, spectral.py:161-195: diag(V^H a_x V) from the products
            dek_dk = -sum((1j * n) * np.einsum("...rm,...rm->...m", vs.conj(), p) * ws ** n
                          for p, n in zip(prods, (-1, 0, 1)))
            ks = -1j * np.log(ws)
        dek_dk = np.nan_to_num(dek_dk, nan=0, posinf=0, neginf=0)
        ks = np.nan_to_num(ks, nan=0, posinf=0, neginf=0)
        eps = np.finfo(dek_dk.dtype).eps
        ratio = abs(dek_dk.real) / (abs(dek_dk.imag) + eps)
        mask_propagating = np.abs(ks.imag) < self.min_decay
        mask_propagating &= self.min_propagation < ratio
        mask_propagating &= dek_dk.real < 0
        mask_decaying = ks.imag < -self.min_decay
        mask_decaying |= (self.min_propagation >= ratio) & (ks.imag < -self.eta_decay)
        mask_decaying &= ks.imag > -self.max_decay
        return (mask_propagating | mask_decaying) & (residuals < self.residual_tolerance)

    def solve_device(self, a_ii: torch.Tensor, a_ij: torch.Tensor, a_ji: torch.Tensor):
        """(B, b, b) device stacks in; (x_ii, reflected-mode mask) out."""
        batch, b = a_ii.shape[0], a_ii.shape[-1]
        device = a_ii.device
        ws, vs = self.nevp((a_ji, a_ii, a_ij))
        ws = ws.reshape(batch, -1)
        vs = vs.reshape(batch, b, -1)
        with np.errstate(divide="ignore", invalid="ignore"):
            vs = vs / np.linalg.norm(vs, axis=-2, keepdims=True)  # _upscale_eigenmodes
        m0 = vs.shape[-1]
        vd = torch.from_numpy(np.ascontiguousarray(vs)).to(device)
        prods = [_zgemm(a, vd, torch.empty((batch, b, m0), dtype=_C128, device=device)).cpu().numpy()
                 for a in (a_ji, a_ii, a_ij)]
        mask = self._find_reflected_modes(ws, vs, prods)
        # _compute_x_ii, spectral.py:349-390: x_ii a_ij = (V_r / w) pinv(V_r),
        # a rank-m product formed on the GPU from padded host factors.
        left = np.zeros((batch, b, m0), dtype=np.complex128)
        right = np.zeros((batch, m0, b), dtype=np.complex128)
        for i in range(batch):
            m = mask[i]
            vr = vs[i][:, m]
            k = vr.shape[1]
            left[i, :, :k] = vr / ws[i][m]
            right[i, :k, :] = np.linalg.inv(vr.conj().T @ vr) @ vr.conj().T
        x_a = _zgemm(torch.from_numpy(left).to(device), torch.from_numpy(right).to(device),
                     torch.empty((batch, b, b), dtype=_C128, device=device))
        x = inverse(_zgemm(a_ji, x_a, torch.empty_like(a_ii), addend=a_ii))
        for _ in range(self.num_ref_iterations - 1):  # spectral.py:574-576
            x, _, _ = fixed_point_refine(a_ii, a_ij, a_ji, x)
        x, _, _ = fixed_point_refine(a_ii, a_ij, a_ji, x)  # spectral.py:627
        return x, mask

    def __call__(self, a_ii, a_ij, a_ji, contact: str, return_injected: bool = False,
                 return_modes_only: bool = False):
        """spectral.py:392-629: the surface Green's function x_ii."""
        if return_injected or return_modes_only:
            raise NotImplementedError("the injection vectors of the wave-function solver are not provided")
        device = self.device or default_device()
        like = a_ii
        shape = tuple(a_ii.shape)
        x, _ = self.solve_device(_dev3(a_ii, device), _dev3(a_ij, device), _dev3(a_ji, device))
        return from_device(x.reshape(shape), like)
