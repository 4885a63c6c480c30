"""Open-boundary conditions with the qttools OBC plugin interface.

* ``OBCSolver`` / ``SanchoRubio`` mirror
  ``src/qttools/boundary_conditions/obc/obc.py:11-49`` and
  ``src/qttools/boundary_conditions/obc/sancho_rubio.py:12-85``.
* ``OBCSystem`` mirrors the memoizing wrapper
  ``src/qttools/boundary_conditions/obc/obc.py:52-202`` with
  ``BaseBoundarySystem`` (``boundary_conditions/boundary_system.py:48-373``):
  memoization modes, residual test, refinement steps and warnings.
* ``contact_self_energy`` is the boundary self-energy glue of
  ``src/quatrex/electron/solver.py:483-489``; ``transmission`` is the Caroli
  formula evaluated from G^R_{0,N-1}.

All arithmetic runs in libqtx_b200; arrays may be NumPy, CuPy or torch and
results come back in the caller's array type.
"""

from __future__ import annotations

import ctypes
import warnings
from abc import ABC, abstractmethod

import numpy as np
import torch

from . import _native
from ._interop import default_device, from_device, kind, mat, stack3, to_device
from .utils import workspace_pool


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _dev3(x, device) -> torch.Tensor:
    return stack3(to_device(x, device)).contiguous()


class OBCSolver(ABC):
    """Surface Green's function x_ii = (a_ii - a_ji x_ii a_ij)^{-1}."""

    @abstractmethod
    def __call__(self, a_ii, a_ij, a_ji, contact: str):
        ...


class SanchoRubio(OBCSolver):
    """Sancho-Rubio decimation on the GPU.

    Parameters
    ----------
    max_iterations : int
        Maximum decimation steps (reference default 100).
    convergence_tol : float
        Stop when ||(|alpha| + |beta|)||_F / 2 < tol (reference default 1e-6).
    per_energy : bool
        False (default): one batch-wide stop, as the reference does
        (sancho_rubio.py:73-78). True: every energy stops as soon as its own
        measure is below the tolerance; converged energies do no further
        work.
    """

    def __init__(self, max_iterations: int = 100, convergence_tol: float = 1e-6,
                 per_energy: bool = False, device: torch.device | None = None):
        self.max_iterations = max_iterations
        self.convergence_tol = convergence_tol
        self.per_energy = per_energy
        self.device = device
        self.last_iterations = 0

    def solve_device(self, a_ii: torch.Tensor, a_ij: torch.Tensor, a_ji: torch.Tensor,
                     out: torch.Tensor | None = None) -> tuple[torch.Tensor, int, bool]:
        """Device tensors (B, n, n) in, (x, iterations, converged) out."""
        lib = _native.load()
        device = a_ii.device
        batch, n = a_ii.shape[0], a_ii.shape[-1]
        x = torch.empty_like(a_ii) if out is None else out
        ws = workspace_pool.get(lib.qtx_sancho_rubio_workspace(n, batch), device, "sr")
        info = torch.zeros(batch, dtype=torch.int32, device=device)
        it, conv = ctypes.c_int(0), ctypes.c_int(0)
        _native.check(lib.qtx_sancho_rubio(n, batch, mat(a_ii), mat(a_ij), mat(a_ji), mat(x),
                                           int(self.max_iterations), float(self.convergence_tol),
                                           int(self.per_energy), ctypes.byref(it), ctypes.byref(conv),
                                           None, info.data_ptr(), ws.data_ptr(), ws.numel(),
                                           _stream(device)))
        self.last_iterations = it.value
        return x, it.value, bool(conv.value)

    def __call__(self, a_ii, a_ij, a_ji, contact: str):
        device = self.device or default_device()
        shape = tuple(a_ii.shape)
        x, _, conv = self.solve_device(_dev3(a_ii, device), _dev3(a_ij, device), _dev3(a_ji, device))
        if not conv:
            warnings.warn("Surface Green's function did not converge.", RuntimeWarning)
        return from_device(x.reshape(shape), a_ii)


def fixed_point_refine(a_ii: torch.Tensor, a_ij: torch.Tensor, a_ji: torch.Tensor, x: torch.Tensor,
                       out: torch.Tensor | None = None):
    """x_ref = inv(a_ii - a_ji x a_ij) with its residuals (obc.py:105-195).
    Device tensors (B, n, n); returns (x_ref, rel_res, abs_res)."""
    lib = _native.load()
    device = x.device
    batch, n = x.shape[0], x.shape[-1]
    x_ref = torch.empty_like(x) if out is None else out
    rel = torch.empty(batch, dtype=torch.float64, device=device)
    ab = torch.empty(batch, dtype=torch.float64, device=device)
    ws = workspace_pool.get(lib.qtx_obc_workspace(n, batch), device, "obc")
    info = torch.zeros(batch, dtype=torch.int32, device=device)
    _native.check(lib.qtx_obc_refine(n, batch, mat(a_ii), mat(a_ij), mat(a_ji), mat(x), mat(x_ref),
                                     rel.data_ptr(), ab.data_ptr(), info.data_ptr(), ws.data_ptr(),
                                     ws.numel(), _stream(device)))
    return x_ref, rel, ab


def inverse(a: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Batched inverse on the GPU (replaces kernels/linalg/inv.py)."""
    lib = _native.load()
    a3 = stack3(a).contiguous()
    x = torch.empty_like(a3) if out is None else out
    info = torch.zeros(a3.shape[0], dtype=torch.int32, device=a3.device)
    _native.check(lib.qtx_zinv_batched(a3.shape[-1], a3.shape[0], mat(a3), mat(x), info.data_ptr(),
                                       _stream(a3.device)))
    if bool((info != 0).any()):
        raise np.linalg.LinAlgError("Singular matrix")
    return x.reshape(a.shape)


class IdentityReducer:
    """System reducer that leaves the boundary system unchanged
    (boundary_conditions/system_reduction.py)."""

    def contract_system(self, system):
        return system

    def expand_solution(self, system, reduced_system, solution):
        return solution

    def expand_residuals(self, system, reduced_system, rel, ab):
        return rel, ab


class OBCSystem:
    """Memoizing OBC wrapper with the semantics of qttools ``OBCSystem``.

    ``__call__((a_ii, a_ij, a_ji), contact)`` returns
    ``(x, rel_residuals, abs_residuals)``. The cache keeps device copies of
    the last solution per contact (warm starts stay resident on the GPU).
    ``stack_comm`` is an optional ``torch.distributed`` process group used
    for the cross-rank agreement of the "auto" mode
    (boundary_system.py:280-296); on one rank it is the identity.
    """

    def __init__(self, boundary_solver: OBCSolver, cache_compressor=None, system_reducer=None,
                 num_ref_iterations: int = 2, relative_tol: float = 2e-1, absolute_tol: float = 1e-6,
                 warning_threshold: float = 1e-1, memoization_mode: str = "auto",
                 agreement_threshold: float = 0.999, stack_comm=None, device=None):
        self.boundary_solver = boundary_solver
        self.num_ref_iterations = num_ref_iterations
        self.relative_tol = relative_tol
        self.absolute_tol = absolute_tol
        self.warning_threshold = warning_threshold
        self.memoization_mode = memoization_mode
        self.agreement_threshold = agreement_threshold
        self.stack_comm = stack_comm
        self.device = device
        if cache_compressor is not None:
            if not hasattr(cache_compressor, "compress"):
                raise ValueError("Cache compressor must have a 'compress' method.")
            if not hasattr(cache_compressor, "decompress"):
                raise ValueError("Cache compressor must have a 'decompress' method.")
        self.cache_compressor = cache_compressor
        if not (0.0 <= self.agreement_threshold <= 1.0):
            raise ValueError("Memoizing tolerance must be between 0 and 1.")
        self.system_reducer = system_reducer or IdentityReducer()
        for attr in ("contract_system", "expand_solution", "expand_residuals"):
            if not hasattr(self.system_reducer, attr):
                raise ValueError(f"System reducer must have a '{attr}' method.")
        self._cache: dict = {}
        if self.num_ref_iterations < 2:
            warnings.warn("The number of refinement iterations should be at least 2. Defaulting to 2.",
                          RuntimeWarning)
            self.num_ref_iterations = 2

    # -- cache -----------------------------------------------------------
    def _compress(self, x):
        return self.cache_compressor.compress(x) if self.cache_compressor else x.clone()

    def _decompress(self, x):
        if x is None:
            return None
        return self.cache_compressor.decompress(x) if self.cache_compressor else x

    # -- steps -----------------------------------------------------------
    def _fixed_point_step(self, system, solution):
        a_ii, a_ij, a_ji = system
        x, _, _ = fixed_point_refine(a_ii, a_ij, a_ji, solution)
        return x

    def _get_starting_guess(self, system):
        return inverse(system[0])

    def _get_residuals(self, system, test_solution):
        a_ii, a_ij, a_ji = system
        x, rel, ab = fixed_point_refine(a_ii, a_ij, a_ji, test_solution)
        return rel, ab, x

    def _solve(self, system, contact):
        if isinstance(self.boundary_solver, SanchoRubio):
            solution, _, conv = self.boundary_solver.solve_device(*system)
            if not conv:
                warnings.warn("Surface Green's function did not converge.", RuntimeWarning)
        else:
            solution = _dev3(self.boundary_solver(*system, contact), system[0].device)
        if self.memoization_mode != "off":
            self._cache[contact] = self._compress(solution)
        return solution

    def _memoized_solve(self, system, contact):
        if self.memoization_mode == "off":
            return self._solve(system, contact)
        solution = self._decompress(self._cache.get(contact, None))
        if solution is None:
            if self.memoization_mode in ("auto", "force-after-first"):
                return self._solve(system, contact)
            elif self.memoization_mode == "force":
                solution = self._get_starting_guess(system)
            else:
                raise RuntimeError(f"Invalid memoizing mode: {self.memoization_mode}")
        rel, ab, solution = self._get_residuals(system, solution)
        if self.memoization_mode == "auto":
            local = int(((ab < self.absolute_tol) | (rel < self.relative_tol)).sum().item())
            total = torch.tensor([local], dtype=torch.int64, device=rel.device)
            size = 1
            if self.stack_comm is not None:
                import torch.distributed as dist  # noqa: PLC0415

                dist.all_reduce(total, group=self.stack_comm)
                size = dist.get_world_size(self.stack_comm)
            if total.item() / size > self.agreement_threshold:
                return self._solve(system, contact)
        for _ in range(self.num_ref_iterations - 2):
            solution = self._fixed_point_step(system, solution)
        return solution

    def __call__(self, boundary_system, contact: str):
        device = self.device or default_device()
        like = boundary_system[0]
        shape = tuple(like.shape)
        system = tuple(_dev3(a, device) for a in boundary_system)
        reduced = self.system_reducer.contract_system(system)
        sol = self._memoized_solve(reduced, contact)
        rel, ab, sol = self._get_residuals(reduced, sol)
        if bool(((rel > self.warning_threshold) & (ab > self.absolute_tol)).any()):
            warnings.warn(
                f"High error for {contact} of OBCSolver {type(self.boundary_solver).__name__}:\n"
                f"  Relative recursion error: {rel.max().item():.3e}\n"
                f"  Absolute recursion error: {ab.max().item():.3e}\n", RuntimeWarning)
        if self.memoization_mode != "off":
            self._cache[contact] = self._compress(sol)
        sol = self.system_reducer.expand_solution(system, reduced, sol)
        rel, ab = self.system_reducer.expand_residuals(system, reduced, rel, ab)
        lead = shape[:-2]
        return (from_device(sol.reshape(shape), like), from_device(rel.reshape(lead), like),
                from_device(ab.reshape(lead), like))


def contact_self_energy(a_ij, a_ji, g, occupancies=None, device=None):
    """Boundary self-energies of a contact (electron/solver.py:483-489):
    sigma = a_ji g a_ij; lesser = i f Gamma; greater = i (f - 1) Gamma with
    Gamma = i (sigma - sigma^H). Returns (sigma, lesser, greater); the last
    two are None without occupancies."""
    lib = _native.load()
    device = device or default_device()
    shape = tuple(g.shape)
    G = _dev3(g, device)
    batch, n = G.shape[0], G.shape[-1]
    Aij, Aji = _dev3(a_ij, device), _dev3(a_ji, device)
    sig = torch.empty_like(G)
    sl = sg = None
    occ_t = None
    if occupancies is not None:
        occ_t = to_device(occupancies, device, dtype=torch.float64).reshape(-1).contiguous()
        sl, sg = torch.empty_like(G), torch.empty_like(G)
    ws = workspace_pool.get(lib.qtx_obc_workspace(n, batch), device, "obc")
    _native.check(lib.qtx_contact_self_energy(
        n, batch, mat(Aij), mat(Aji), mat(G), occ_t.data_ptr() if occ_t is not None else None, mat(sig),
        mat(sl), mat(sg), ws.data_ptr(), ws.numel(), _stream(device)))
    res = [from_device(sig.reshape(shape), g)]
    res += [from_device(t.reshape(shape), g) if t is not None else None for t in (sl, sg)]
    return tuple(res)


def transmission(g0n, sigma_left, sigma_right, device=None):
    """Caroli transmission Tr[Gamma_L G_{0,N-1} Gamma_R G_{0,N-1}^H]."""
    lib = _native.load()
    device = device or default_device()
    G = _dev3(g0n, device)
    SL, SR = _dev3(sigma_left, device), _dev3(sigma_right, device)
    batch, m, n = G.shape
    t = torch.empty(batch, dtype=torch.float64, device=device)
    ws = workspace_pool.get(lib.qtx_obc_workspace(max(m, n), batch), device, "obc")
    _native.check(lib.qtx_transmission(m, n, batch, mat(G), mat(SL), mat(SR), t.data_ptr(), ws.data_ptr(),
                                       ws.numel(), _stream(device)))
    return from_device(t.reshape(tuple(g0n.shape[:-2])), g0n) if kind(g0n) != "torch" else t.reshape(
        tuple(g0n.shape[:-2]))
