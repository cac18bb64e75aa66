"""Batched unbinding of isolated NFW halos given as a list input (one region
per halo; the batched-unbinding workload at reduced size): FoF bit-exact,
unbinding within the FP32 tolerance of the oracle."""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native, workloads as W
from tests.helpers import oracle_core

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
    assert np.array_equal(g[0], o[0])
    assert np.array_equal(g[1], o[1])


@pytest.mark.parametrize("fp64", [True, False])
def test_nfw_list_unbinding(fp64):
    sizes = [30, 55, 120, 400, 800, 1500, 2600, 5000, 12000, 25] * 3
    xs, vs = W.nfw_halos(len(sizes), seed=3, sizes=sizes)
    kw = dict(vp_list=vs, L_Box=512.0, linking_length=0.2, np_halo_min=10, bound_check=True)
    _native.set_option("unbind_fp64", int(fp64))
    try:
        g = P._fof_core(xs, **kw)
    finally:
        _native.set_option("unbind_fp64", 0)
    o = oracle_core(xs, **kw)
    n_in = int(o[0].sum())
    assert n_in > 1000
    assert _native.get_stat("pm_halos") >= 1
    mism = int((g[0] != o[0]).sum())
    assert mism <= max(3, n_in // 1000), (mism, n_in)
    assert abs(int(g[1].max()) - int(o[1].max())) <= 1
