"""The plugin on qttools' own ``DSDBCOO`` containers (NumPy backend).

``tests/golden/make_qttools_containers.py`` built qttools ``DSDBCOO``
objects with the reference package and recorded the attributes the plugin
reads, together with the ``data`` that the reference's ``RGF.selected_solve``
(``src/qttools/greens_function_solver/rgf.py:115-438``) and
``RGF.selected_inv`` (``rgf.py:25-113``) wrote into fresh
``DSDBCOO.zeros_like`` outputs. Here containers with those attributes (the
class is named ``DSDBCOO`` and holds NumPy host arrays, like the reference's
NumPy-backed one) go through ``quatrex_b200.RGF``; the nonzeros it writes,
in qttools' block-sorted order, must match the reference's at the FP64
parity gate (1e-10 relative).
"""

import numpy as np
import pytest

from quatrex_b200 import RGF, OBCBlocks

pytestmark = pytest.mark.gpu


class DSDBCOO:
    """A NumPy-backed container with the recorded qttools DSDBCOO attributes
    (``src/qttools/datastructures/dsdbcoo.py``, ``dsdbsparse.py:140-240``)."""

    def __init__(self, data, rows, cols, block_sizes, global_stack_shape, symmetry=False):
        self.data = data
        self.rows = rows
        self.cols = cols
        self.block_sizes = block_sizes
        self.num_blocks = len(block_sizes)
        self.global_stack_shape = tuple(int(s) for s in global_stack_shape)
        self.symmetry = bool(symmetry)
        n = int(np.sum(block_sizes))
        self.stack_shape = data.shape[:-1]
        self.shape = self.stack_shape + (n, n)

    @classmethod
    def zeros_like(cls, other):
        return cls(np.zeros_like(other.data), other.rows, other.cols, other.block_sizes,
                   other.global_stack_shape, other.symmetry)


def _container(g, name):
    m = DSDBCOO(g[f"{name}_data"].copy(), g[f"{name}_rows"], g[f"{name}_cols"], g[f"{name}_block_sizes"],
                g[f"{name}_global_stack_shape"], bool(g[f"{name}_symmetry"]))
    assert m.shape == tuple(g[f"{name}_shape"]) and m.num_blocks == int(g[f"{name}_num_blocks"])
    return m


def _obc(g, n):
    obc = OBCBlocks(num_blocks=n)
    for key in ("retarded", "lesser", "greater"):
        getattr(obc, key)[0] = g[f"obc_{key}_first"]
        getattr(obc, key)[-1] = g[f"obc_{key}_last"]
    return obc


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def fixture(golden):
    return golden("qttools_dsdbcoo")


def test_selected_solve_on_qttools_containers(cuda_device, fixture):
    g = fixture
    a, sl, sg = (_container(g, k) for k in ("a", "sigma_lesser", "sigma_greater"))
    obc = _obc(g, a.num_blocks)
    xl, xg, xr = RGF(max_batch_size=2).selected_solve(a, sl, sg, obc_blocks=obc, return_retarded=True)
    for name, x in (("xl", xl), ("xg", xg), ("xr", xr)):
        assert type(x).__name__ == "DSDBCOO" and isinstance(x.data, np.ndarray)
        np.testing.assert_array_equal(x.rows, g[f"{name}_rows"])
        ref = g[f"{name}_data"]
        # same nonzero order, same values (nonzeros the reference leaves at zero stay zero)
        np.testing.assert_array_equal(x.data == 0, ref == 0)
        assert _rel(x.data, ref) < 1e-10, (name, _rel(x.data, ref))


def test_selected_solve_out_and_current_on_qttools_containers(cuda_device, fixture):
    g = fixture
    a, sl, sg = (_container(g, k) for k in ("a", "sigma_lesser", "sigma_greater"))
    outs = tuple(DSDBCOO.zeros_like(a) for _ in range(3))
    current = RGF(max_batch_size=5).selected_solve(a, sl, sg, obc_blocks=_obc(g, a.num_blocks), out=outs,
                                                   return_retarded=True, return_current=True)
    assert _rel(np.asarray(current), g["current"]) < 1e-10
    for name, x in zip(("xl", "xg", "xr"), outs):
        assert _rel(x.data, g[f"{name}_data"]) < 1e-10, name
    with pytest.raises(ValueError):
        RGF().selected_solve(a, sl, sg, out=outs[:1])


def test_selected_inv_on_qttools_containers(cuda_device, fixture):
    g = fixture
    a = _container(g, "a")
    x = RGF(max_batch_size=3).selected_inv(a, obc_blocks=_obc(g, a.num_blocks))
    assert _rel(x.data, g["inv_data"]) < 1e-10
    out = DSDBCOO.zeros_like(a)
    assert RGF(max_batch_size=2).selected_inv(a, obc_blocks=_obc(g, a.num_blocks), out=out) is None
    assert _rel(out.data, g["inv_data"]) < 1e-10
