"""Boundary conditions of the screened interaction W: the Lyapunov solver
interface and its doubling solver, the memoizing Lyapunov system, and the
contact glue of the Coulomb-screening solve.

* ``LyapunovSolver`` / ``Doubling`` mirror
  ``src/qttools/boundary_conditions/lyapunov/lyapunov.py:10-49`` and
  ``lyapunov/doubling.py:9-91`` (``qtx_lyapunov_doubling``);
* ``LyapunovSystem`` mirrors ``lyapunov.py:424-579`` on the memoizer of
  ``OBCSystem`` (``boundary_system.py:200-373``), with the fixed-point step
  x = q + a x a^H (``qtx_lyapunov_refine``) and q as the starting guess;
* ``screened_contact_obc`` is ``CoulombScreeningSolver._compute_contact_obc``
  (``src/quatrex/coulomb_screening/solver.py:211-378``) for
  ``block_sections = 1`` and one connected block: the retarded, lesser and
  greater boundary self-energies of W from the boundary blocks of the
  retarded / lesser / greater polarization and of the Coulomb matrix, with
  every product on the GPU.
"""

from __future__ import annotations

import ctypes
import warnings
from abc import ABC, abstractmethod

import numpy as np
import torch

from . import _native
from ._interop import default_device, from_device, mat, stack3, to_device
from .obc import OBCSystem, _stream
from .utils import workspace_pool

_C128 = torch.complex128
_NULL = _native.NULL_MAT


def _zgemm(a, b, out, op_a=0, op_b=0, addend=None, alpha=1.0, beta=1.0):
    """out = alpha op(a) op(b) (+ beta addend), batched (B, n, n) device stacks."""
    lib = _native.load()
    batch, n = a.shape[0], a.shape[-1]
    _native.check(lib.qtx_zgemm_batched(n, n, n, batch, alpha, 0.0, mat(a), op_a, mat(b), op_b, beta, 0.0,
                                        mat(addend) if addend is not None else _NULL, 0, mat(out),
                                        _stream(a.device)))
    return out


def _mm(a, b, op_a=0, op_b=0):
    return _zgemm(a, b, torch.empty(a.shape, dtype=_C128, device=a.device), op_a, op_b)


def _flat(a, q):
    """(a, q) as contiguous (S, n, n) device stacks, a broadcast to q's shape."""
    n = q.shape[-1]
    return torch.broadcast_to(a, q.shape).reshape(-1, n, n).contiguous(), q.reshape(-1, n, n).contiguous()


class LyapunovSolver(ABC):
    """Solver of the discrete-time Lyapunov equation x = q + a x a^H."""

    @abstractmethod
    def __call__(self, a, q, contact: str):
        ...


class Doubling(LyapunovSolver):
    """Doubling solver of the Lyapunov equation (``doubling.py:9-91``):
    x_{k+1} = x_k + a_k x_k a_k^H, a_{k+1} = a_k^2, stopped when every entry
    meets the relative or the absolute tolerance; a RuntimeWarning when
    ``max_iterations`` is reached first."""

    def __init__(self, max_iterations: int = 10, convergence_rel_tol: float = 1e-5,
                 convergence_abs_tol: float = 1e-8, device: torch.device | None = None) -> None:
        self.max_iterations = max_iterations
        self.convergence_rel_tol = convergence_rel_tol
        self.convergence_abs_tol = convergence_abs_tol
        self.device = device
        self.last_iterations = 0

    def solve_device(self, a: torch.Tensor, q: torch.Tensor) -> tuple[torch.Tensor, bool]:
        """Device tensors in (q.ndim >= a.ndim, broadcast); (x, converged) out."""
        lib = _native.load()
        af, qf = _flat(a, q)
        batch, n = qf.shape[0], qf.shape[-1]
        x = torch.empty_like(qf)
        ws = workspace_pool.get(lib.qtx_lyapunov_workspace(n, batch), qf.device, "lyapunov")
        it, conv = ctypes.c_int(0), ctypes.c_int(0)
        _native.check(lib.qtx_lyapunov_doubling(n, batch, mat(af), mat(qf), mat(x), int(self.max_iterations),
                                                float(self.convergence_rel_tol), float(self.convergence_abs_tol),
                                                ctypes.byref(it), ctypes.byref(conv), ws.data_ptr(), ws.numel(),
                                                _stream(qf.device)))
        self.last_iterations = it.value
        return x.reshape(q.shape), bool(conv.value)

    def __call__(self, a, q, contact: str):
        if tuple(q.shape[-2:]) != tuple(a.shape[-2:]) or q.ndim < a.ndim:
            raise AssertionError("q must have a's matrix shape and at least its dimensions")
        device = self.device or default_device()
        x, conv = self.solve_device(to_device(a, device), to_device(q, device))
        if not conv:
            warnings.warn("The doubling method for the Lyapunov equation did not converge.", RuntimeWarning)
        return from_device(x, q)


def lyapunov_refine(a: torch.Tensor, q: torch.Tensor, x: torch.Tensor):
    """x_ref = q + a x a^H with its residuals (lyapunov.py:488-579); device
    tensors, a broadcast to q's shape. Returns (x_ref, rel, abs)."""
    lib = _native.load()
    af, qf = _flat(a, q)
    xf = x.reshape(qf.shape).contiguous()
    batch, n = qf.shape[0], qf.shape[-1]
    x_ref = torch.empty_like(qf)
    rel = torch.empty(batch, dtype=torch.float64, device=qf.device)
    ab = torch.empty(batch, dtype=torch.float64, device=qf.device)
    ws = workspace_pool.get(lib.qtx_lyapunov_workspace(n, batch), qf.device, "lyapunov")
    _native.check(lib.qtx_lyapunov_refine(n, batch, mat(af), mat(qf), mat(xf), mat(x_ref), rel.data_ptr(),
                                          ab.data_ptr(), ws.data_ptr(), ws.numel(), _stream(qf.device)))
    lead = tuple(q.shape[:-2])
    return x_ref.reshape(q.shape), rel.reshape(lead), ab.reshape(lead)


class LyapunovSystem(OBCSystem):
    """Memoizing Lyapunov system (``lyapunov.py:424-579``): the memoization
    modes, agreement rule, refinement steps and warnings of ``OBCSystem``
    with the Lyapunov fixed point x = q + a x a^H. Called as
    ``system((a, q), contact) -> (x, rel_residuals, abs_residuals)``."""

    def __init__(self, boundary_solver: LyapunovSolver, cache_compressor=None, system_reducer=None,
                 num_ref_iterations: int = 2, relative_tol: float = 2e-1, absolute_tol: float = 1e-6,
                 warning_threshold: float = 1e-1, memoization_mode: str = "auto",
                 agreement_threshold: float = 0.999, stack_comm=None, device=None):
        super().__init__(boundary_solver, cache_compressor, system_reducer, num_ref_iterations, relative_tol,
                         absolute_tol, warning_threshold, memoization_mode, agreement_threshold, stack_comm,
                         device)

    def _fixed_point_step(self, system, solution):
        a, q = system
        x, _, _ = lyapunov_refine(a, q, solution)
        return x

    def _get_starting_guess(self, system):
        return system[1].clone()

    def _get_residuals(self, system, test_solution):
        a, q = system
        x, rel, ab = lyapunov_refine(a, q, test_solution)
        return rel, ab, x

    def _solve(self, system, contact):
        a, q = system
        if isinstance(self.boundary_solver, Doubling):
            solution, conv = self.boundary_solver.solve_device(a, q)
            if not conv:
                warnings.warn("The doubling method for the Lyapunov equation did not converge.", RuntimeWarning)
        else:
            solution = to_device(self.boundary_solver(a, q, contact), q.device)
        if self.memoization_mode != "off":
            self._cache[contact] = self._compress(solution)
        return solution

    def __call__(self, boundary_system, contact: str):
        device = self.device or default_device()
        a, q = boundary_system
        like = q
        system = (to_device(a, device).contiguous(), to_device(q, device).contiguous())
        reduced = self.system_reducer.contract_system(system)
        sol = self._memoized_solve(reduced, contact)
        rel, ab, sol = self._get_residuals(reduced, sol)
        if bool(((rel > self.warning_threshold) & (ab > self.absolute_tol)).any()):
            warnings.warn(
                f"High error for {contact} of LyapunovSolver {type(self.boundary_solver).__name__}:\n"
                f"  Relative recursion error: {rel.max().item():.3e}\n"
                f"  Absolute recursion error: {ab.max().item():.3e}\n", RuntimeWarning)
        if self.memoization_mode != "off":
            self._cache[contact] = self._compress(sol)
        sol = self.system_reducer.expand_solution(system, reduced, sol)
        rel, ab = self.system_reducer.expand_residuals(system, reduced, rel, ab)
        return from_device(sol, like), from_device(rel, like), from_device(ab, like)


def screened_contact_obc(p_retarded, p_lesser, p_greater, v, obc, lyapunov, contact: str = "left",
                         device: torch.device | None = None):
    """Retarded, lesser and greater boundary self-energies of the screened
    interaction for one contact (``coulomb_screening/solver.py:260-378``,
    block_sections = 1, one connected block). Each of ``p_retarded``,
    ``p_lesser``, ``p_greater`` and ``v`` is the triple (x_10, x_00, x_01) of
    boundary blocks in the left-contact order ((B, n, n) stacks, or (n, n)
    for the energy-independent Coulomb matrix); ``obc`` is an ``OBCSystem``
    (any OBC solver) and ``lyapunov`` a ``LyapunovSystem``. Results come
    back in the array type of ``p_retarded``."""
    device = device or default_device()
    like = p_retarded[1]
    batch = stack3(to_device(p_retarded[1], device)).shape[0]

    def d3(x):
        t = stack3(to_device(x, device))
        if t.shape[0] != batch:
            t = t.expand(batch, -1, -1)
        return t.contiguous()

    p10, p00, p01 = (d3(x) for x in p_retarded)
    v10, v00, v01 = (d3(x) for x in v)
    n = p00.shape[-1]
    eye = torch.eye(n, dtype=_C128, device=device).expand(batch, n, n).contiguous()
    # m blocks (solver.py:273-280): m_00 = I - v10 p01 - v00 p00 - v01 p10, ...
    m_00 = _zgemm(v01, p10, torch.empty_like(p00), alpha=-1.0,
                  addend=_zgemm(v00, p00, torch.empty_like(p00), alpha=-1.0,
                                addend=_zgemm(v10, p01, torch.empty_like(p00), alpha=-1.0, addend=eye)))
    m_01 = _zgemm(v01, p00, torch.empty_like(p00), alpha=-1.0,
                  addend=_zgemm(v00, p01, torch.empty_like(p00), alpha=-1.0))
    m_10 = _zgemm(v00, p10, torch.empty_like(p00), alpha=-1.0,
                  addend=_zgemm(v10, p00, torch.empty_like(p00), alpha=-1.0))
    x_00, _, _ = obc((m_00, m_01, m_10), contact="W: " + contact)
    x_00 = to_device(x_00, device).reshape(batch, n, n).contiguous()
    m_10_x_00 = _mm(m_10, x_00)
    obc_retarded = _mm(m_10_x_00, m_01)

    def l_superblocks(p_):  # solver.py:307-335
        """l_00 = sum of the 7 and l_01 of the 5 products v_a q v_b the
        reference lists, grouped by the left Coulomb factor:
        l_00 = v10 s1 + v00 s3 + v01 s4 and l_01 = v10 q01 v01 + v00 s1 + v01 s2
        with the inner sums s1 = q00 v01 + q01 v00, s2 = q10 v01 + q00 v00,
        s3 = s2 + q01 v10 and s4 = q10 v00 + q00 v10, which both blocks share:
        14 batched products instead of 24."""
        q10, q00, q01 = (d3(x) for x in p_)

        def e():
            return torch.empty_like(p00)

        s1 = _zgemm(q01, v00, e(), addend=_mm(q00, v01))
        s2 = _zgemm(q00, v00, e(), addend=_mm(q10, v01))
        s3 = _zgemm(q01, v10, e(), addend=s2)
        s4 = _zgemm(q00, v10, e(), addend=_mm(q10, v00))
        l_00 = _zgemm(v01, s4, e(), addend=_zgemm(v00, s3, e(), addend=_mm(v10, s1)))
        l_01 = _zgemm(v01, s2, e(), addend=_zgemm(v00, s1, e(), addend=_mm(v10, _mm(q01, v01))))
        return l_00, l_01

    out = []
    qs = []
    for p_ in (p_lesser, p_greater):
        l_00, l_01 = l_superblocks(p_)
        a_00 = _mm(m_10_x_00, l_01)  # solver.py:346-347
        anti = a_00 - a_00.conj().transpose(-2, -1)
        inner = (l_00 - anti).contiguous()
        qs.append(_zgemm(_mm(x_00, inner), x_00, torch.empty_like(p00), op_b=1))
        out.append(anti)
    b_00 = _mm(x_00, m_10)
    q_00 = torch.stack(qs)
    w_00, _, _ = lyapunov((b_00, q_00), contact="W: " + contact)
    w_00 = to_device(w_00, device).reshape(2, batch, n, n)
    obc_lg = []
    for k in range(2):
        mw = _mm(m_10, w_00[k].contiguous())
        m_w_m = _zgemm(mw, m_10, torch.empty_like(p00), op_b=1)
        obc_lg.append(m_w_m - out[k])
    shape = tuple(like.shape)
    return tuple(from_device(t.reshape(shape), like) for t in (obc_retarded, obc_lg[0], obc_lg[1]))
