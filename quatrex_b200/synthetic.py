"""Seeded synthetic transport devices for the NEGF hot path.

The device is a block-tridiagonal tight-binding Hamiltonian with ``N``
diagonal blocks of size ``b``:

* ``H_ii = (M_i + M_i^H) / 2`` with ``M_i = (X + iY) / 8`` and X, Y standard
  normal ``b x b`` draws;
* one coupling ``T = (X + iY) / 8`` shared by every ``(i, i+1)`` pair, with
  ``H_{i+1,i} = T^H``.

Draw order (``numpy.random.default_rng(seed)``): for ``i = 0..N-1`` the real
part then the imaginary part of ``M_i``; then the real part then the
imaginary part of ``T``. The leads repeat the first and last block pair, so
the open-boundary blocks are taken from the system matrix itself (the
``block_sections == 1`` case of qttools' ``get_periodic_superblocks``,
``src/qttools/toeplitz/toeplitz.py:76-77``).

The system matrix at energy ``E`` is ``A(E) = (E + i eta) I - H`` and the
contact occupations follow the Fermi function ``f(x) = 1 / (1 + exp(x/kT))``
with ``f_L(E) = f(E)``, ``f_R(E) = f(E - bias)``
(``src/quatrex/core/statistics.py:7-23``).

Configurations (sizes of the reference benchmark workloads):

=====  ====  ====  =========  ==============
name    N     b    energies    energy window
=====  ====  ====  =========  ==============
cfg0    16    64       32       [-2, 2]
cfg1    32   256     1024       [-3, 3]
cfg2    64   512     2048       [-3, 3]
=====  ====  ====  =========  ==============
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

ETA = 1e-4
KT = 0.025
BIAS = 0.1


@dataclass
class Device:
    """A block-tridiagonal device Hamiltonian (host, complex128)."""

    h_diag: np.ndarray  # (N, b, b)
    coupling: np.ndarray  # (b, b): block (i, i+1); block (i+1, i) is its adjoint
    energies: np.ndarray  # (E,)
    eta: float = ETA
    kT: float = KT
    bias: float = BIAS
    name: str = "custom"
    meta: dict = field(default_factory=dict)

    @property
    def num_blocks(self) -> int:
        return int(self.h_diag.shape[0])

    @property
    def block_size(self) -> int:
        return int(self.h_diag.shape[1])

    @property
    def block_sizes(self) -> np.ndarray:
        return np.full(self.num_blocks, self.block_size, dtype=np.int64)

    def fermi_left(self, energies: np.ndarray | None = None) -> np.ndarray:
        e = self.energies if energies is None else np.asarray(energies)
        return fermi(e, self.kT)

    def fermi_right(self, energies: np.ndarray | None = None) -> np.ndarray:
        e = self.energies if energies is None else np.asarray(energies)
        return fermi(e - self.bias, self.kT)

    def system_blocks(self, energies: np.ndarray | None = None):
        """Dense blocks of ``A(E) = (E + i eta) I - H`` for the given energies.

        Returns ``(diag, upper, lower)`` lists: ``diag[i]`` has shape
        ``(E, b, b)``; ``upper[i]`` is block ``(i, i+1)``; ``lower[i]`` is
        block ``(i+1, i)``.
        """
        e = self.energies if energies is None else np.asarray(energies)
        z = (e + 1j * self.eta).astype(np.complex128)
        b = self.block_size
        eye = np.eye(b, dtype=np.complex128)
        diag = [z[:, None, None] * eye - self.h_diag[i][None] for i in range(self.num_blocks)]
        up = np.broadcast_to(-self.coupling, (e.size, b, b)).copy()
        lo = np.broadcast_to(-self.coupling.conj().T, (e.size, b, b)).copy()
        upper = [up.copy() for _ in range(self.num_blocks - 1)]
        lower = [lo.copy() for _ in range(self.num_blocks - 1)]
        return diag, upper, lower

    def dense_hamiltonian(self) -> np.ndarray:
        n, b = self.num_blocks, self.block_size
        h = np.zeros((n * b, n * b), dtype=np.complex128)
        for i in range(n):
            h[i * b:(i + 1) * b, i * b:(i + 1) * b] = self.h_diag[i]
            if i + 1 < n:
                h[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = self.coupling
                h[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = self.coupling.conj().T
        return h


def fermi(x: np.ndarray, kT: float) -> np.ndarray:
    """Fermi-Dirac occupation ``1 / (1 + exp(x / kT))`` (x in eV)."""
    return 1.0 / (1.0 + np.exp(np.asarray(x, dtype=np.float64) / kT))


def make_device(num_blocks: int, block_size: int, energies: np.ndarray, seed: int = 0,
                name: str = "custom") -> Device:
    """Builds the seeded random device described in the module docstring."""
    rng = np.random.default_rng(seed)
    b = int(block_size)
    h = np.empty((num_blocks, b, b), dtype=np.complex128)
    for i in range(num_blocks):
        re = rng.standard_normal((b, b))
        im = rng.standard_normal((b, b))
        m = (re + 1j * im) / 8.0
        h[i] = 0.5 * (m + m.conj().T)
    re = rng.standard_normal((b, b))
    im = rng.standard_normal((b, b))
    t = (re + 1j * im) / 8.0
    return Device(h_diag=h, coupling=t, energies=np.asarray(energies, dtype=np.float64), name=name)


def cfg0() -> Device:
    """16 blocks of 64x64, 32 energies uniform in [-2, 2], seed 0."""
    return make_device(16, 64, np.linspace(-2.0, 2.0, 32), seed=0, name="cfg0")


def cfg1(num_energies: int = 1024) -> Device:
    """32 blocks of 256x256, 1024 energies uniform in [-3, 3], seed 0."""
    return make_device(32, 256, np.linspace(-3.0, 3.0, num_energies), seed=0, name="cfg1")


def cfg2(num_energies: int = 2048) -> Device:
    """64 blocks of 512x512, 2048 energies uniform in [-3, 3], seed 0."""
    return make_device(64, 512, np.linspace(-3.0, 3.0, num_energies), seed=0, name="cfg2")


def uneven_devices(num_devices: int = 8, num_energies: int = 256, seed: int = 1,
                   block_counts=(8, 16, 32, 64), block_sizes=(128, 256, 384, 512, 768)):
    """The uneven batch: per device, N then b drawn uniformly with
    ``default_rng(seed)``; each device is then built like :func:`cfg0` (seed
    0 Hamiltonian construction with its own N, b) on ``num_energies`` energies
    uniform in [-2, 2]."""
    rng = np.random.default_rng(seed)
    shapes = []
    for _ in range(num_devices):
        n = int(rng.choice(block_counts))
        b = int(rng.choice(block_sizes))
        shapes.append((n, b))
    return shapes


def random_bt_dense(block_sizes, seed: int = 0, density: float = 0.5) -> np.ndarray:
    """Quasi-sparse, diagonally dominant random block-tridiagonal matrix.

    Same construction as the qttools GF-solver test fixture
    (``tests/qttools/greens_function_solver/conftest.py:58-104``), with a
    seeded generator so the case is reproducible.
    """
    rng = np.random.default_rng(seed)
    block_sizes = np.asarray(block_sizes, dtype=np.int64)
    offs = np.concatenate(([0], np.cumsum(block_sizes)))
    size = int(offs[-1])
    arr = np.zeros((size, size), dtype=np.complex128)

    def rblock(m, n):
        mask = rng.random((m, n)) < density
        vals = rng.random((m, n)) + 1j * rng.random((m, n))
        return np.where(mask, vals, 0.0)

    for i in range(len(block_sizes)):
        arr[offs[i]:offs[i + 1], offs[i]:offs[i + 1]] = rblock(block_sizes[i], block_sizes[i]) + np.eye(
            block_sizes[i])
        if i > 0:
            arr[offs[i]:offs[i + 1], offs[i - 1]:offs[i]] = rblock(block_sizes[i], block_sizes[i - 1])
            arr[offs[i - 1]:offs[i], offs[i]:offs[i + 1]] = rblock(block_sizes[i - 1], block_sizes[i])
    for i in range(size):
        arr[i, i] = (1 + 1j) + arr[i, :].sum()
    return arr


def strip_lead(width: int, slices: int, energies, seed: int = 0, eta: float = ETA, disorder: float = 0.3):
    """Boundary blocks of a semi-infinite strip lead: a square lattice
    ``width`` sites wide with nearest-neighbour hopping -1, onsite energies
    uniform in [-disorder/2, disorder/2] (``default_rng(seed)``), cut into
    blocks of ``slices`` consecutive slices (block size width x slices).
    Returns ``(a_ii, a_ij, a_ji)`` of ``A = (E + i eta) I - H`` as
    (E, b, b) complex128 stacks. The coupling between blocks has rank
    ``width``, so at most 2 x width of the 2 b eigenmodes of the lead are
    finite and nonzero, and only the propagating and slowly decaying ones lie
    in an annulus around the unit circle: the regime that contour-integral
    (Beyn) OBC solvers with a subspace of a few modes are built for."""
    rng = np.random.default_rng(seed)
    b = width * slices
    h = np.diag(rng.uniform(-disorder / 2, disorder / 2, b)).astype(np.complex128)
    for s_ in range(slices):
        for c in range(width - 1):
            i = s_ * width + c
            h[i, i + 1] = h[i + 1, i] = -1.0
        if s_ + 1 < slices:
            for c in range(width):
                i = s_ * width + c
                h[i, i + width] = h[i + width, i] = -1.0
    t = np.zeros((b, b), dtype=np.complex128)  # H_{i,i+1}: last slice -> next block's first slice
    for c in range(width):
        t[(slices - 1) * width + c, c] = -1.0
    e = np.asarray(energies, dtype=np.float64)
    z = (e + 1j * eta)[:, None, None]
    eye = np.eye(b, dtype=np.complex128)
    a_ii = z * eye - h
    a_ij = np.broadcast_to(-t, (e.size, b, b)).copy()
    a_ji = np.broadcast_to(-t.conj().T, (e.size, b, b)).copy()
    return a_ii, a_ij, a_ji


def screened_lead(block_size: int, num_energies: int, seed: int = 0):
    """Boundary blocks of a synthetic screened-interaction (W) problem: the
    Coulomb matrix V (Hermitian, positive definite diagonal block, weak
    coupling) and the retarded, lesser and greater polarization P^R, P^<,
    P^> of ``num_energies`` energies, with the symmetries the reference
    relies on (P^< = i X, P^> = -i Y with X, Y positive semidefinite
    block-tridiagonal; P^R with a dissipative anti-Hermitian part).
    Returns dicts of (x_10, x_00, x_01) triples: ``v`` of (b, b) blocks and
    ``p_retarded``, ``p_lesser``, ``p_greater`` of (E, b, b) stacks."""
    rng = np.random.default_rng(seed)
    b, ne = int(block_size), int(num_energies)

    def cplx(*s):
        return rng.standard_normal(s) + 1j * rng.standard_normal(s)

    def h(x):
        return x.conj().swapaxes(-2, -1)

    u, _ = np.linalg.qr(cplx(b, b))
    v00 = (u * rng.uniform(0.2, 1.0, b)) @ h(u) * 0.5
    v01 = 0.05 * cplx(b, b)
    v = (h(v01), v00, v01)
    herm = 0.5 * (cplx(ne, b, b) + h(cplx(ne, b, b)))
    g = cplx(ne, b, b)
    p00 = 0.04 * herm - 0.02j * (g @ h(g)) / b
    p01 = 0.01 * cplx(ne, b, b)
    p10 = 0.01 * cplx(ne, b, b)
    out = {"v": v, "p_retarded": (p10, p00, p01)}
    for name, sign in (("p_lesser", 1.0), ("p_greater", -1.0)):
        q0, q1 = cplx(ne, b, b) * 0.1, cplx(ne, b, b) * 0.05
        x00 = q0 @ h(q0) + q1 @ h(q1)
        x01 = q1 @ h(q0)
        out[name] = (1j * sign * h(x01), 1j * sign * x00, 1j * sign * x01)
    return out


def screened_device(num_blocks: int, block_size: int, num_energies: int, seed: int = 0,
                    interior: float = 0.3):
    """Block-tridiagonal inputs of a synthetic screened-interaction (W) solve
    in small blocks: the Coulomb matrix V (Hermitian; positive definite
    diagonal blocks, weak coupling) and, for ``num_energies`` energies, the
    lesser and greater polarization P^< = i X, P^> = -i Y (X, Y positive
    semidefinite: X = Q Q^H with Q block lower bidiagonal) and the Hermitian
    part P^R_h of the retarded polarization. The first two and the last two
    blocks repeat one periodic lead cell (the contacts' boundary blocks);
    the blocks in between are the lead's blocks perturbed by ``interior``
    relative random parts. Returns a dict with ``v`` = (diag, upper, lower)
    lists of (b, b) blocks and ``p_lesser``, ``p_greater``,
    ``p_retarded_hermitian`` = (diag, upper, lower) lists of (E, b, b)
    stacks (upper[i] = block (i, i+1), lower[i] = block (i+1, i))."""
    rng = np.random.default_rng(seed)
    n, b, ne = int(num_blocks), int(block_size), int(num_energies)

    def cplx(*s):
        return rng.standard_normal(s) + 1j * rng.standard_normal(s)

    def h(x):
        return x.conj().swapaxes(-2, -1)

    def lead_or_interior(i, lead, draw):
        # blocks 0, 1 and n-2, n-1 belong to the contacts' periodic cells
        if i <= 1 or i >= n - 2:
            return lead
        return lead * (1.0 + interior * draw())

    u, _ = np.linalg.qr(cplx(b, b))
    v00 = (u * rng.uniform(0.2, 1.0, b)) @ h(u) * 0.5
    v01 = 0.05 * cplx(b, b)
    v_diag = [v00.copy() for _ in range(n)]
    v_upper = [lead_or_interior(i, v01, lambda: rng.uniform()) for i in range(n - 1)]
    v_lower = [h(x) for x in v_upper]
    herm = 0.5 * (cplx(ne, b, b) + h(cplx(ne, b, b)))
    p_diag = [lead_or_interior(i, 0.04 * herm, lambda: rng.uniform()) for i in range(n)]
    p_up = 0.01 * cplx(ne, b, b)
    p_upper = [lead_or_interior(i, p_up, lambda: rng.uniform()) for i in range(n - 1)]
    p_lower = [h(x) for x in p_upper]
    out = {"v": (v_diag, v_upper, v_lower), "p_retarded_hermitian": (p_diag, p_upper, p_lower)}
    for name, sign in (("p_lesser", 1.0), ("p_greater", -1.0)):
        q0, q1 = cplx(ne, b, b) * 0.1, cplx(ne, b, b) * 0.05
        qd = [lead_or_interior(i, q0, lambda: rng.uniform()) for i in range(n)]
        qs = [lead_or_interior(i, q1, lambda: rng.uniform()) for i in range(n)]  # Q[i, i-1] = qs[i]
        xd = [qd[i] @ h(qd[i]) + qs[i] @ h(qs[i]) for i in range(n)]
        xl = [qs[i + 1] @ h(qd[i]) for i in range(n - 1)]  # X[i+1, i]
        xu = [h(x) for x in xl]
        out[name] = ([1j * sign * x for x in xd], [1j * sign * x for x in xu], [1j * sign * x for x in xl])
    return out
