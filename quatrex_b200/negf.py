"""The per-energy NEGF unit of work on resident device data.

One *energy point* is what ``ElectronSolver.solve``
(``src/quatrex/electron/solver.py:756-888``) does per energy with zero
scattering self-energy:

1. assemble ``A(E) = (E + i eta) I - H`` (solver.py:668-709);
2. both contacts: Sancho-Rubio surface Green's function
   (``qttools/boundary_conditions/obc/sancho_rubio.py:33-85``) followed by the
   ``OBCSystem`` residual/refinement step (``boundary_system.py:303-373``),
   then ``Sigma = a_ji g a_ij``, ``Sigma^< = i f Gamma``,
   ``Sigma^> = i (f - 1) Gamma`` (solver.py:420-495);
3. ``RGF.selected_solve`` for G^R, G^<, G^> with the Meir-Wingreen current
   (``qttools/greens_function_solver/rgf.py:115-438``);
4. the Caroli transmission and the density Im diag G^<
   (``quatrex/core/observables.py:8-31``).

The Hamiltonian blocks stay resident on the GPU; energy-independent blocks
(the couplings and the zero scattering self-energy blocks) are single
blocks shared by the whole batch (stack stride 0), and every product is
still executed as in the general solver. Output block stacks are allocated
once per batch size and reused.
"""

from __future__ import annotations

import ctypes
import warnings
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from ._interop import mat
from ._native import NULL_MAT, QtxBT, QtxMat
from .emulation import gemm_path
from .obc import SanchoRubio
from .utils import WorkspacePool

_C128 = torch.complex128


def _bcast(t: torch.Tensor) -> QtxMat:
    """A single (b, b) block seen as a stack with stride 0."""
    return QtxMat(t.data_ptr(), t.shape[-1], 0)


@dataclass
class ScatteringSelfEnergy:
    """Scattering self-energies of one batch, as the electron solve of an
    SCBA iteration receives them (quatrex electron/solver.py:756-888):
    ``retarded`` (its Hermitian part), ``lesser`` and ``greater`` are each
    ``(diag, upper, lower)`` device complex128 stacks of shapes (N, B, b, b),
    (N-1, B, b, b), (N-1, B, b, b), or None for zero."""

    retarded: tuple | None = None
    lesser: tuple | None = None
    greater: tuple | None = None


@dataclass
class PointResult:
    transmission: torch.Tensor  # (B,) float64
    density: torch.Tensor  # (B, N*b) float64
    current: torch.Tensor  # (B, N+1) complex128
    sigma_left: torch.Tensor
    sigma_right: torch.Tensor
    sr_iterations: tuple
    blocks: dict = field(default_factory=dict)


class EnergyPointSolver:
    """Solves batches of energy points of one block-tridiagonal device.

    Parameters
    ----------
    h_diag : (N, b, b) complex array
        Diagonal Hamiltonian blocks.
    coupling : (b, b) complex array
        Block (i, i+1) of H; block (i+1, i) is its adjoint.
    eta : float
        Broadening in ``A = (E + i eta) I - H``.
    sr_tol, sr_max_iterations : Sancho-Rubio stop criterion.
    per_energy : bool
        Per-energy Sancho-Rubio convergence (converged energies stop
        iterating) instead of the batch-wide stop.
    skip_zero_scattering : bool
        False (default): the zero scattering self-energy is passed as zero
        blocks and every product of the general solve is executed, as in the
        reference. True: it is passed as absent and the products with it are
        skipped (ballistic shortcut).
    device_loop : bool
        Run Sancho-Rubio with device-side convergence (no host
        synchronisation; required for CUDA-graph capture). The host-driven
        loop (default) stops at exactly the reference's iteration.
    precision : "fp64", "mixed" or "emulated"
        "fp64": complex128 throughout (FP64 DMMA products).
        "emulated": complex128 throughout; the products of the selected
        solve are formed on the int8 tensor cores from ``slices`` digit
        planes per operand (``emulation.py``; ~1e-12 relative per product at
        6 slices, FP64 level at 7). The boundary conditions stay on FP64
        DMMA products: the Sancho-Rubio doubling recursion amplifies product
        errors by orders of magnitude.
        "mixed": the boundary conditions (Sancho-Rubio, refinement, contact
        self-energies) stay FP64; the selected solve stores complex64 blocks
        and runs its products on tcgen05 as split-TF32 products with FP32
        accumulation, inverting every Schur complement in FP64; the
        transmission is formed in FP64 from the complex64 corner block.
    potential : (N, b) real array, optional
        Electrostatic potential per orbital, subtracted on the diagonal of
        A(E) like ``ElectronSolver._assemble_system_matrix``
        (``electron/solver.py:668-709``, potential at :701); the leads use the
        potential of their edge blocks.
    store_blocks : bool
        True (default): the G^<, G^> (diagonal and off-diagonal) and G^R
        diagonal blocks of the last batch are kept in ``PointResult.blocks``.
        False: only the observables (transmission, density, current) are
        produced; the solve writes no output blocks, which roughly halves the
        device memory per energy.
    """

    def __init__(self, h_diag, coupling, eta: float = 1e-4, sr_tol: float = 1e-12,
                 sr_max_iterations: int = 100, per_energy: bool = True,
                 skip_zero_scattering: bool = False, device: torch.device | None = None,
                 precision: str = "fp64", device_loop: bool = False, store_blocks: bool = True,
                 potential=None, slices: int = 6):
        if precision not in ("fp64", "mixed", "emulated"):
            raise ValueError(f"precision must be 'fp64', 'mixed' or 'emulated', got {precision!r}")
        if precision == "emulated" and not 3 <= int(slices) <= 8:
            raise ValueError(f"slices must be 3-8, got {slices}")
        self.precision = precision
        # GEMM path of the library calls: 0 = FP64 DMMA, else int8 emulation
        self.slices = int(slices) if precision == "emulated" else 0
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        h = torch.as_tensor(np.asarray(h_diag), dtype=_C128) if not isinstance(h_diag, torch.Tensor) else h_diag
        t = torch.as_tensor(np.asarray(coupling), dtype=_C128) if not isinstance(coupling, torch.Tensor) else coupling
        self.h = h.to(self.device, _C128).contiguous()
        if potential is not None:
            # A_ii = (E + i eta) I - H_ii - diag(V_i): the energy-independent
            # potential is folded into the resident diagonal blocks once.
            v = torch.as_tensor(np.asarray(potential, dtype=np.float64)).to(self.device)
            if v.shape != self.h.shape[:2]:
                raise ValueError(f"potential must have shape {tuple(self.h.shape[:2])}, got {tuple(v.shape)}")
            self.h = self.h + torch.diag_embed(v.to(_C128))
        self.N, self.b = int(self.h.shape[0]), int(self.h.shape[-1])
        self.upper = (-t).to(self.device, _C128).contiguous()
        self.lower = (-t.conj().transpose(-2, -1)).to(self.device, _C128).contiguous()
        self.zero = torch.zeros((self.b, self.b), dtype=_C128, device=self.device)
        if precision == "mixed":
            self.upper64 = self.upper.to(torch.complex64)
            self.lower64 = self.lower.to(torch.complex64)
            self.zero64 = torch.zeros((self.b, self.b), dtype=torch.complex64, device=self.device)
        self.eta = float(eta)
        self.sr = SanchoRubio(max_iterations=sr_max_iterations, convergence_tol=sr_tol,
                              per_energy=per_energy)
        self.skip_zero_scattering = skip_zero_scattering
        self.device_loop = device_loop
        self.store_blocks = store_blocks
        self._bufs: dict = {}
        self._graphs: dict = {}
        self._host_sr = (0, True)
        self._last_device_loop = device_loop
        # Workspaces belong to this solver: captured graphs hold their
        # addresses, and solvers on concurrent streams must not share them.
        self._ws = WorkspacePool()
        self._grid = None  # (energies, f_left, f_right) on the device, see bind_grid
        self._cache = None  # resident surface Green's functions, see enable_obc_cache
        self._scatt = None  # scattering self-energies of the current eager call
        self._h_off = None
        self.lib = _native.load()

    # ------------------------------------------------------------------
    def bind_grid(self, energies, f_left, f_right) -> None:
        """Keeps an energy grid (with lead occupations) on the device. A batch
        is then named by grid indices (:meth:`set_indices`) and the captured
        pipeline gathers its energies itself, so one replay needs only the
        index vector as input."""
        dev = self.device
        as_dev = lambda x: torch.as_tensor(np.asarray(x, dtype=np.float64)).reshape(-1).to(dev)  # noqa: E731
        self._grid = (as_dev(energies), as_dev(f_left), as_dev(f_right))
        self._bufs.clear()
        self._graphs.clear()

    def enable_obc_cache(self) -> None:
        """Resident warm starts: the refined surface Green's functions of
        every grid energy solved so far stay on the device (two b x b blocks
        per grid point). A warm run reads them instead of running
        Sancho-Rubio and applies the OBCSystem fixed-point step
        (``boundary_system.py:303-373``) to them."""
        if self._grid is None:
            raise RuntimeError("enable_obc_cache() needs bind_grid() first")
        G = int(self._grid[0].numel())
        z = lambda: torch.zeros((G, self.b, self.b), dtype=_C128, device=self.device)  # noqa: E731
        self._cache = (z(), z())
        self._graphs.clear()

    def cache_bytes(self) -> int:
        return 0 if self._grid is None else 2 * int(self._grid[0].numel()) * self.b * self.b * 16

    def set_indices(self, idx) -> int:
        """Grid indices of the next batch (see bind_grid)."""
        t = torch.as_tensor(np.asarray(idx, dtype=np.int64)).reshape(-1)
        B = int(t.numel())
        self._buffers(B)["idx"].copy_(t)
        return B

    def resident_bytes(self, B: int) -> int:
        """Device bytes this solver holds for batch size B (buffers and
        workspaces), without allocating anything."""
        return resident_bytes(self.N, self.b, B, self.precision, self.lib, self.store_blocks, self.slices)

    def _buffers(self, B: int) -> dict:
        buf = self._bufs.get(B)
        if buf is not None:
            return buf
        N, b, dev = self.N, self.b, self.device
        z = lambda *s: torch.empty(s, dtype=_C128, device=dev)  # noqa: E731
        ot = torch.complex64 if self.precision == "mixed" else _C128
        o = lambda *s: torch.empty(s, dtype=ot, device=dev)  # noqa: E731
        n1 = max(N - 1, 1)
        if self.store_blocks:
            outs = dict(xl_d=o(N, B, b, b), xl_u=o(n1, B, b, b), xl_l=o(n1, B, b, b), xg_d=o(N, B, b, b),
                        xg_u=o(n1, B, b, b), xg_l=o(n1, B, b, b), xr_d=o(N, B, b, b))
        else:
            outs = {}
        buf = dict(
            a_diag=z(N, B, b, b), g0n=o(B, b, b), **outs,
            gl=z(B, b, b), gr=z(B, b, b), sig=[z(B, b, b) for _ in range(6)],
            current=z(B, N + 1), density=torch.empty((B, N * b), dtype=torch.float64, device=dev),
            T=torch.empty(B, dtype=torch.float64, device=dev), zE=z(B),
            info=torch.zeros(B, dtype=torch.int32, device=dev),
            E=torch.empty(B, dtype=torch.float64, device=dev), fl=torch.empty(B, dtype=torch.float64, device=dev),
            fr=torch.empty(B, dtype=torch.float64, device=dev),
            res_rel=[torch.empty(B, dtype=torch.float64, device=dev) for _ in range(2)],
            res_abs=[torch.empty(B, dtype=torch.float64, device=dev) for _ in range(2)],
            sr_it=torch.zeros(1, dtype=torch.int32, device=dev), sr_conv=torch.zeros(1, dtype=torch.int32, device=dev),
        )
        if self._grid is not None:
            buf["idx"] = torch.zeros(B, dtype=torch.int64, device=dev)
        if self.precision == "mixed":
            buf["a_diag64"] = o(N, B, b, b)
            buf["sig64"] = [o(B, b, b) for _ in range(6)]
            buf["g0n128"] = z(B, b, b)
        if self._bufs:
            self._graphs.clear()  # graphs refer to the buffers being replaced
        self._bufs = {B: buf}  # keep one batch size resident
        return buf

    def _bt(self, diag, upper, lower, keep):
        n = self.N
        bs = (ctypes.c_int32 * n)(*([self.b] * n))
        d = (QtxMat * n)(*diag)
        u = (QtxMat * max(n - 1, 1))(*(upper or [NULL_MAT]))
        lo = (QtxMat * max(n - 1, 1))(*(lower or [NULL_MAT]))
        keep.extend([bs, d, u, lo])
        return QtxBT(n, bs, d, u, lo)

    # ------------------------------------------------------------------
    def solve(self, energies, f_left, f_right, scattering: ScatteringSelfEnergy | None = None) -> PointResult:
        """Solves one batch of energies; all results stay on the device.

        ``scattering``: scattering self-energies of the batch (an SCBA
        iteration). The system matrix is then assembled in one pass per block
        as A = (E + i eta) I - V - H - Sigma^R - (Sigma^> - Sigma^<) / 2
        (``qtx_assemble_system``, electron/solver.py:611-709), the boundary
        conditions are taken from the assembled boundary blocks, and
        Sigma^<, Sigma^> enter the selected solve (solver.py:845-872).
        FP64 and emulated precisions; eager calls only (not captured)."""
        B = self.set_inputs(energies, f_left, f_right)
        if scattering is not None:
            if self.precision == "mixed":
                raise NotImplementedError("scattering self-energies are taken by the fp64 and emulated paths")
            self._check_scattering(scattering, B)
        self._scatt = scattering
        try:
            res = self._run(B, device_loop=self.device_loop)
        finally:
            self._scatt = None
        if not self.device_loop:
            it, conv = self._host_sr
            if not conv:
                warnings.warn("Surface Green's function did not converge.", RuntimeWarning)
        return res

    def set_inputs(self, energies, f_left, f_right) -> int:
        """Copies one batch's energies and occupations into the solver's
        device input buffers (the only per-batch host-to-device traffic)."""
        if self._grid is not None:
            raise RuntimeError("this solver is bound to an energy grid: name batches with set_indices()")
        dev = self.device
        E = torch.as_tensor(np.asarray(energies, dtype=np.float64)).reshape(-1)
        B = int(E.numel())
        buf = self._buffers(B)
        buf["E"].copy_(E, non_blocking=False)
        buf["fl"].copy_(torch.as_tensor(np.asarray(f_left, dtype=np.float64)).reshape(-1))
        buf["fr"].copy_(torch.as_tensor(np.asarray(f_right, dtype=np.float64)).reshape(-1))
        return B

    def set_inputs_device(self, energies: torch.Tensor, f_left: torch.Tensor, f_right: torch.Tensor) -> int:
        """set_inputs() from device tensors: asynchronous copies on the
        current stream (no host synchronisation)."""
        B = int(energies.numel())
        buf = self._buffers(B)
        buf["E"].copy_(energies.reshape(-1), non_blocking=True)
        buf["fl"].copy_(f_left.reshape(-1), non_blocking=True)
        buf["fr"].copy_(f_right.reshape(-1), non_blocking=True)
        return B

    def capture(self, B: int, warm: bool = False) -> "torch.cuda.CUDAGraph":
        """Captures the whole energy-point pipeline for batch size B in one
        CUDA graph (Sancho-Rubio runs its device-side convergence loop). The
        inputs are read from the solver's device buffers, so a replay after
        set_inputs() solves a new batch. The first capture runs the pipeline
        once eagerly to allocate every buffer outside the capture."""
        g = self._graphs.get((B, warm))
        if g is not None:
            return g
        self._buffers(B)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self._run(B, device_loop=True, warm=warm)
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self._run(B, device_loop=True, warm=warm)
        self._graphs[(B, warm)] = g
        return g

    def solve_graph(self, energies, f_left, f_right) -> PointResult:
        """solve() through the captured CUDA graph of this batch size."""
        B = self.set_inputs(energies, f_left, f_right)
        g = self.capture(B)
        g.replay()
        return self._result(B)

    def _check_scattering(self, sc: ScatteringSelfEnergy, B: int) -> None:
        N, b = self.N, self.b
        for name in ("retarded", "lesser", "greater"):
            t = getattr(sc, name)
            if t is None:
                continue
            shapes = ((N, B, b, b), (N - 1, B, b, b), (N - 1, B, b, b))
            if len(t) != 3 or any(tuple(x.shape) != sh or x.dtype != _C128 or x.device != self.device
                                  or not x.is_contiguous() for x, sh in zip(t, shapes)):
                raise ValueError(f"scattering.{name} must be contiguous complex128 device stacks of shapes "
                                 f"{shapes}")

    def _assembled(self, B: int, buf: dict, keep: list, stream):
        """A(E) with the scattering self-energies: diagonal blocks into
        a_diag, off-diagonal blocks into per-energy stacks."""
        N, b, lib = self.N, self.b, self.lib
        if buf.get("a_up") is None or buf["a_up"].shape[1] != B:
            n1 = max(N - 1, 1)
            buf["a_up"] = torch.empty((n1, B, b, b), dtype=_C128, device=self.device)
            buf["a_lo"] = torch.empty((n1, B, b, b), dtype=_C128, device=self.device)
        if getattr(self, "_h_off", None) is None:
            self._h_off = ((-self.upper).contiguous(), (-self.lower).contiguous())  # H_{i,i+1}, H_{i+1,i}
        H = self._bt([_bcast(self.h[i]) for i in range(N)], [_bcast(self._h_off[0])] * (N - 1),
                     [_bcast(self._h_off[1])] * (N - 1), keep)
        A = self._bt([mat(buf["a_diag"][i]) for i in range(N)], [mat(buf["a_up"][i]) for i in range(N - 1)],
                     [mat(buf["a_lo"][i]) for i in range(N - 1)], keep)

        def bt(t):
            if t is None:
                return None
            return ctypes.byref(self._bt([mat(t[0][i]) for i in range(N)], [mat(t[1][i]) for i in range(N - 1)],
                                         [mat(t[2][i]) for i in range(N - 1)], keep))

        sc = self._scatt
        _native.check(lib.qtx_assemble_system(ctypes.byref(H), None, buf["zE"].data_ptr(), bt(sc.retarded),
                                              bt(sc.lesser), bt(sc.greater), ctypes.byref(A), B, stream))
        return mat(buf["a_up"][0]), mat(buf["a_lo"][0]), mat(buf["a_up"][N - 2]), mat(buf["a_lo"][N - 2])

    def sr_status(self, B: int) -> tuple[int, bool]:
        """(decimation steps, converged) of the last device-loop run."""
        buf = self._buffers(B)
        return int(buf["sr_it"].item()), bool(buf["sr_conv"].item())

    def _result(self, B: int) -> PointResult:
        buf = self._bufs[B]
        sig = buf["sig"]
        if self.store_blocks:
            blocks = dict(xl_diag=buf["xl_d"], xl_upper=buf["xl_u"], xl_lower=buf["xl_l"], xg_diag=buf["xg_d"],
                          xg_upper=buf["xg_u"], xg_lower=buf["xg_l"], xr_diag=buf["xr_d"], g0n=buf["g0n"])
        else:
            blocks = dict(g0n=buf["g0n"])
        its = (self._host_sr[0],) * 2 if not self._last_device_loop else ("device", "device")
        return PointResult(buf["T"], buf["density"], buf["current"], sig[0], sig[3], its, blocks)

    def _run(self, B: int, device_loop: bool, warm: bool = False) -> PointResult:
        """The kernel sequence of one batch; no host transfers, and no host
        synchronisation when device_loop is set (graph-capturable)."""
        with gemm_path(0):  # FP64 DMMA unless a step below selects the emulation
            return self._enqueue(B, device_loop, warm)

    def _enqueue(self, B: int, device_loop: bool, warm: bool) -> PointResult:
        lib, dev = self.lib, self.device
        N, b = self.N, self.b
        buf = self._bufs[B]
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        keep: list = []
        self._last_device_loop = device_loop
        fl, fr = buf["fl"], buf["fr"]
        if self._grid is not None:  # the batch is named by grid indices
            idx = buf["idx"]
            torch.index_select(self._grid[0], 0, idx, out=buf["E"])
            torch.index_select(self._grid[1], 0, idx, out=fl)
            torch.index_select(self._grid[2], 0, idx, out=fr)
        _native.check(lib.qtx_assemble_energies(B, buf["E"].data_ptr(), float(self.eta), buf["zE"].data_ptr(),
                                                stream))

        # 1. A(E): diagonal blocks (energy-independent couplings stay shared),
        #    or every block when scattering self-energies are given.
        a_diag = buf["a_diag"]
        scatt = getattr(self, "_scatt", None)
        if scatt is None:
            for i in range(N):
                _native.check(lib.qtx_assemble_diag(b, B, _bcast(self.h[i]), buf["zE"].data_ptr(),
                                                    mat(a_diag[i]), stream))
            up0, lo0 = up_n, lo_n = _bcast(self.upper), _bcast(self.lower)
        else:
            up0, lo0, up_n, lo_n = self._assembled(B, buf, keep, stream)

        # 2. Boundary conditions, left = (A00, A01, A10), right =
        #    (A_NN, A_N,N-1, A_N-1,N).
        sig = buf["sig"]
        sides = ((a_diag[0], up0, lo0, buf["gl"], fl, sig[0:3]),
                 (a_diag[N - 1], lo_n, up_n, buf["gr"], fr, sig[3:6]))
        if warm:
            if self._cache is None:
                raise RuntimeError("a warm run needs enable_obc_cache()")
            torch.index_select(self._cache[0], 0, buf["idx"], out=buf["gl"])
            torch.index_select(self._cache[1], 0, buf["idx"], out=buf["gr"])
        else:
            self._sr_both(sides, B, stream, device_loop, buf)
        for k, (aii, aij, aji, g, f, s3) in enumerate(sides):
            ws = self._ws.get(lib.qtx_obc_workspace(b, B), dev, "obc")
            _native.check(lib.qtx_obc_refine(b, B, mat(aii), aij, aji, mat(g), mat(g),
                                             buf["res_rel"][k].data_ptr(), buf["res_abs"][k].data_ptr(), None,
                                             ws.data_ptr(), ws.numel(), stream))
            _native.check(lib.qtx_contact_self_energy(b, B, aij, aji, mat(g), f.data_ptr(), mat(s3[0]),
                                                      mat(s3[1]), mat(s3[2]), ws.data_ptr(), ws.numel(),
                                                      stream))
        if self._cache is not None:
            self._cache[0].index_copy_(0, buf["idx"], buf["gl"])
            self._cache[1].index_copy_(0, buf["idx"], buf["gr"])
        self.last_residuals = (torch.maximum(buf["res_rel"][0], buf["res_rel"][1]) if not device_loop
                               else buf["res_rel"][0], buf["res_abs"][0])

        # 3. Selected solve.
        mixed = self.precision == "mixed"
        if mixed:
            for i in range(N):
                _native.check(lib.qtx_convert(b, b, B, mat(a_diag[i]), _native.QTX_C128,
                                              mat(buf["a_diag64"][i]), _native.QTX_C64, stream))
            for k in range(6):
                _native.check(lib.qtx_convert(b, b, B, mat(sig[k]), _native.QTX_C128, mat(buf["sig64"][k]),
                                              _native.QTX_C64, stream))
            ad, sgx = buf["a_diag64"], buf["sig64"]
            up_s, lo_s, zero = _bcast(self.upper64), _bcast(self.lower64), self.zero64
        else:
            ad, sgx = a_diag, sig
            up_s, lo_s, zero = _bcast(self.upper), _bcast(self.lower), self.zero
        if scatt is None:
            A = self._bt([mat(ad[i]) for i in range(N)], [up_s] * (N - 1), [lo_s] * (N - 1), keep)
        else:
            A = self._bt([mat(ad[i]) for i in range(N)], [mat(buf["a_up"][i]) for i in range(N - 1)],
                         [mat(buf["a_lo"][i]) for i in range(N - 1)], keep)
        zs = NULL_MAT if self.skip_zero_scattering else _bcast(zero)
        S = self._bt([zs] * N, [zs] * (N - 1), [zs] * (N - 1), keep)

        def scatt_bt(t):
            if t is None:
                return S
            return self._bt([mat(t[0][i]) for i in range(N)], [mat(t[1][i]) for i in range(N - 1)],
                            [mat(t[2][i]) for i in range(N - 1)], keep)

        SL = scatt_bt(scatt.lesser) if scatt is not None else S
        SG = scatt_bt(scatt.greater) if scatt is not None else S
        if self.store_blocks:
            XL = self._bt([mat(buf["xl_d"][i]) for i in range(N)], [mat(buf["xl_u"][i]) for i in range(N - 1)],
                          [mat(buf["xl_l"][i]) for i in range(N - 1)], keep)
            XG = self._bt([mat(buf["xg_d"][i]) for i in range(N)], [mat(buf["xg_u"][i]) for i in range(N - 1)],
                          [mat(buf["xg_l"][i]) for i in range(N - 1)], keep)
            XR = self._bt([mat(buf["xr_d"][i]) for i in range(N)], [NULL_MAT] * (N - 1), [NULL_MAT] * (N - 1),
                          keep)
        else:  # observables only: the solve keeps its blocks in its workspace
            XL = self._bt([NULL_MAT] * N, [NULL_MAT] * (N - 1), [NULL_MAT] * (N - 1), keep)
            XG = self._bt([NULL_MAT] * N, [NULL_MAT] * (N - 1), [NULL_MAT] * (N - 1), keep)
            XR = self._bt([NULL_MAT] * N, [NULL_MAT] * (N - 1), [NULL_MAT] * (N - 1), keep)
        obc = []
        for k in range(3):
            arr = (QtxMat * N)(*([NULL_MAT] * N))
            arr[0] = mat(sgx[k])
            arr[N - 1] = mat(sgx[3 + k])
            obc.append(arr)
        wsq = lib.qtx_selected_solve_mixed_workspace if mixed else lib.qtx_selected_solve_workspace
        solve = lib.qtx_selected_solve_mixed if mixed else lib.qtx_selected_solve
        with gemm_path(self.slices):
            ws = self._ws.get(wsq(N, A.block_sizes, B, 1), dev, "rgf")
            _native.check(solve(
                ctypes.byref(A), ctypes.byref(SL), ctypes.byref(SG), obc[0], obc[1], obc[2], ctypes.byref(XL),
                ctypes.byref(XG), ctypes.byref(XR), buf["current"].data_ptr(), mat(buf["g0n"]),
                buf["density"].data_ptr(), 0, B, buf["info"].data_ptr(), ws.data_ptr(), ws.numel(), stream))

        # 4. Transmission (FP64 from the corner block).
        g0n = buf["g0n"]
        if mixed:
            _native.check(lib.qtx_convert(b, b, B, mat(g0n), _native.QTX_C64, mat(buf["g0n128"]),
                                          _native.QTX_C128, stream))
            g0n = buf["g0n128"]
        ws = self._ws.get(lib.qtx_obc_workspace(b, B), dev, "obc")
        _native.check(lib.qtx_transmission(b, b, B, mat(g0n), mat(sig[0]), mat(sig[3]),
                                           buf["T"].data_ptr(), ws.data_ptr(), ws.numel(), stream))
        return self._result(B)

    def _sr_both(self, sides, B: int, stream, device_loop: bool, buf):
        """Both contacts' Sancho-Rubio in one decimation loop (2B entries)."""
        lib, dev = self.lib, self.device
        ws = self._ws.get(lib.qtx_sancho_rubio_workspace(self.b, 2 * B), dev, "sr")
        batches = (ctypes.c_int64 * 2)(B, B)
        aii = (QtxMat * 2)(mat(sides[0][0]), mat(sides[1][0]))
        aij = (QtxMat * 2)(sides[0][1], sides[1][1])
        aji = (QtxMat * 2)(sides[0][2], sides[1][2])
        x = (QtxMat * 2)(mat(sides[0][3]), mat(sides[1][3]))
        if device_loop:
            _native.check(lib.qtx_sancho_rubio_multi_async(
                self.b, 2, batches, aii, aij, aji, x, int(self.sr.max_iterations), float(self.sr.convergence_tol),
                int(self.sr.per_energy), buf["sr_it"].data_ptr(), buf["sr_conv"].data_ptr(), None, ws.data_ptr(),
                ws.numel(), stream))
            return
        it, conv = ctypes.c_int(0), ctypes.c_int(0)
        _native.check(lib.qtx_sancho_rubio_multi(
            self.b, 2, batches, aii, aij, aji, x, int(self.sr.max_iterations), float(self.sr.convergence_tol),
            int(self.sr.per_energy), ctypes.byref(it), ctypes.byref(conv), None, ws.data_ptr(), ws.numel(),
            stream))
        self._host_sr = (it.value, bool(conv.value))


def resident_bytes(N: int, b: int, B: int, precision: str = "fp64", lib=None, store_blocks: bool = True,
                   slices: int = 6) -> int:
    """Device bytes of an EnergyPointSolver(N blocks of b x b) at batch size
    B: the block stacks of EnergyPointSolver._buffers plus the selected-solve,
    Sancho-Rubio and OBC workspaces (sizes from the library's own queries)."""
    lib = lib or _native.load()
    if precision == "emulated":
        bs = (ctypes.c_int32 * N)(*([b] * N))
        with gemm_path(0):
            base = resident_bytes(N, b, B, "fp64", lib, store_blocks)
            plain = int(lib.qtx_selected_solve_workspace(N, bs, B, 1))
        with gemm_path(slices):
            return base - plain + int(lib.qtx_selected_solve_workspace(N, bs, B, 1))
    bb = b * b
    n1 = max(N - 1, 1)
    osz = 8 if precision == "mixed" else 16
    total = 16 * (N * B * bb + 2 * B * bb + 6 * B * bb + B * (N + 1) + B)  # a_diag, g, sigma, current, zE
    total += 8 * (B * N * b + 5 * B) + 4 * (B + 2)  # density, T/E/fl/fr, info, SR status
    total += 16 * 2 * B  # residual vectors
    total += osz * ((3 * N + 4 * n1) * B * bb if store_blocks else 0) + osz * B * bb  # output blocks, corner
    if precision == "mixed":
        total += 8 * (N * B * bb + 6 * B * bb) + 16 * B * bb
    bs = (ctypes.c_int32 * N)(*([b] * N))
    wsq = lib.qtx_selected_solve_mixed_workspace if precision == "mixed" else lib.qtx_selected_solve_workspace
    total += int(wsq(N, bs, B, 1)) + int(lib.qtx_sancho_rubio_workspace(b, 2 * B)) + int(lib.qtx_obc_workspace(b, B))
    return int(total)


def flops_per_energy(N: int, b: int, sr_iterations: tuple = (0, 0)) -> dict:
    """Reference ("as written") real-flop counts of one energy point:
    a complex b x b x b product = 8 b^3 flops, a complex inverse = 8 b^3.

    F_solve = 8b^3 [N + 4 + 33(N-1)]   (rgf.py:234-238,272-301,334-410)
    F_cur   = 8b^3 [9(N-1) + 4]        (rgf.py:389-428)
    F_SR    = 8b^3 [11K + 1] per contact (sancho_rubio.py:64-83)
    F_obc   = 8b^3 [3 + 2] per contact (refinement step + sigma product)
    """
    u = 8.0 * b ** 3
    f_solve = u * (N + 4 + 33 * (N - 1))
    f_cur = u * (9 * (N - 1) + 4)
    f_sr = sum(u * (11 * k + 1) for k in sr_iterations)
    f_obc = 2 * u * 5
    f_trans = u * 2
    return dict(solve=f_solve, current=f_cur, sr=f_sr, obc=f_obc, transmission=f_trans,
                total=f_solve + f_cur + f_sr + f_obc + f_trans)
