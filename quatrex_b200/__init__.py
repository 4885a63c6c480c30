"""quatrex_b200 -- B200 (sm_100a) implementation of QuaTrEx's per-energy
NEGF hot path behind the qttools solver interfaces.

* :class:`RGF` -- drop-in for ``qttools.greens_function_solver.RGF``
  (``selected_inv`` / ``selected_solve``);
* :class:`SanchoRubio`, :class:`Spectral` (with the :class:`Beyn` NEVP
  solver), :class:`OBCSystem` -- drop-ins for the qttools OBC solvers and
  their memoizing wrapper;
* :class:`DSDBCOO` -- torch-backed block-sorted COO stack with the qttools
  block / stack indexers;
* :class:`EnergyPointSolver` -- the whole per-energy unit (OBC + selected
  solve + current + transmission + density) on resident device data;
* :class:`Doubling`, :class:`LyapunovSystem` and
  :class:`CoulombScreeningSolve` -- the screened-interaction (W) boundary
  conditions and solve of a Coulomb-screening step.

All arithmetic runs in ``lib/libqtx_b200.so`` (hand-written CUDA, C ABI in
``include/qtx_b200.h``); there is no CPU fallback.
"""

from .datastructures import DSDBCOO
from .greens_function_solver import RGF, GFSolver, OBCBlocks
from .negf import EnergyPointSolver, ScatteringSelfEnergy, flops_per_energy
from .obc import (OBCSolver, OBCSystem, SanchoRubio, contact_self_energy, fixed_point_refine, inverse,
                  transmission)
from .observables import density
from .spectral import Beyn, Spectral
from .lyapunov import Doubling, LyapunovSolver, LyapunovSystem, screened_contact_obc
from .screening import CoulombScreeningSolve

__all__ = [
    "DSDBCOO", "RGF", "GFSolver", "OBCBlocks", "EnergyPointSolver", "ScatteringSelfEnergy", "flops_per_energy", "OBCSolver",
    "OBCSystem", "SanchoRubio", "contact_self_energy", "fixed_point_refine", "inverse", "transmission",
    "density", "Beyn", "Spectral", "Doubling", "LyapunovSolver", "LyapunovSystem", "screened_contact_obc",
    "CoulombScreeningSolve",
]

__version__ = "0.1.0"
