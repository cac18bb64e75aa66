"""Batched unbinding of isolated NFW halos given as a list input (one region
per halo; the batched-unbinding workload at reduced size): FoF bit-exact,
unbinding within the energy band of the oracle (tests/helpers.py)."""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native, workloads as W
from tests.helpers import check_ang_mom_consistent, check_unbinding_band, oracle_core, oracle_core_diag

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 2])
def test_nfw_list_fof_exact(seed):
    """Very dense centres: cells of one linking length hold hundreds of
    particles and take the warp-cooperative dense path without sub-cells."""
    xs, _ = W.nfw_halos(40, seed=seed, sizes=[20, 60, 300, 2000, 9000, 30000, 150, 40] * 5)
    kw = dict(L_Box=512.0, linking_length=0.2, np_halo_min=10)
    g = P._fof_core(xs, **kw)
    o = oracle_core(xs, **kw)
    assert _native.get_stat("dense_cells") > 0
    assert _native.get_stat("vd_cells") > 0  # NFW cusps: cells linked by merge sub-cells
    assert np.array_equal(g[0], o[0])
    assert np.array_equal(g[1], o[1])


@pytest.mark.parametrize("fp64", [True, False])
def test_nfw_list_unbinding(fp64):
    sizes = [30, 55, 120, 400, 800, 1500, 2600, 5000, 12000, 25] * 3
    xs, vs = W.nfw_halos(len(sizes), seed=3, sizes=sizes)
    kw = dict(vp_list=vs, L_Box=512.0, linking_length=0.2, np_halo_min=10, bound_check=True,
              return_ang_mom=True)
    with _native.options(unbind_fp64=int(fp64)):
        g = P._fof_core(xs, **kw)
    assert _native.get_stat("pm_halos") >= 1
    o, energy, scale = oracle_core_diag(xs, **kw)
    assert int(o[0].sum()) > 1000
    flips, worst = check_unbinding_band(g, o, energy, scale)
    print(f"nfw fp64={fp64}: {flips} flips, worst |E|/max|phi| = {worst:.2e}")
    check_ang_mom_consistent(g, xs, vs, None, 512.0)
