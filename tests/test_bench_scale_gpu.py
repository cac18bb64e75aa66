"""Parity at the benchmark workloads' own sizes and densities.

* fof_256 (16,777,216 particles, the FoF + unbinding box without
  unbinding): the partition bit-exact against the oracle at full size, so
  the dense-cell linking on Plummer cores runs at the density it is timed
  at;
* fof_unbind_128 (2,097,152 particles, a sub-volume of the default bench box
  with the same recipe): FoF bit-exact, unbinding on both precision paths
  within the energy band (tests/helpers.py) with equal halo counts;
* unbind_nfw_2k (2,000 isolated NFW halos up to 200,000 members, the
  batched-unbinding list at a tenth of its size): halos above 32,768
  members take the chunked removal loop.
"""
import numpy as np
import pytest

import bench
import py_fof_b200 as P
from py_fof_b200 import _native
from tests.helpers import (check_ang_mom_consistent, check_unbinding_band, oracle_core,
                           oracle_core_diag)

pytestmark = pytest.mark.gpu


def _kw(wl, bound):
    regions = wl["regions"]
    kw = dict(L_Box=wl["L"], linking_length=bench.LINK, np_halo_min=wl["np_min"],
              ng_global=wl["ng_global"], return_ang_mom=True)
    if bound:
        kw.update(vp_list=wl["vp"] if regions is None else regions[1], mp_list=wl["mp"],
                  bound_check=True, softening=bench.SOFTENING)
    return (wl["xp"] if regions is None else regions[0]), kw


def test_fof_256_bit_exact():
    wl = bench.make_workload("fof_256", 0)
    x, kw = _kw(wl, False)
    g = P._fof_core(x, **kw)
    assert _native.get_stat("dense_cells") > 0
    o = oracle_core(x, **kw)
    assert o[1].max() > 1000
    assert np.array_equal(g[0], o[0])
    assert np.array_equal(g[1], o[1])


@pytest.mark.parametrize("fp64", [1, 0])
def test_fof_unbind_128(fp64):
    wl = bench.make_workload("fof_unbind_128", 0)
    x, kw = _kw(wl, False)
    assert np.array_equal(P._fof_core(x, **kw)[1], oracle_core(x, **kw)[1])
    x, kw = _kw(wl, True)
    with _native.options(unbind_fp64=fp64):
        g = P._fof_core(x, **kw)
    assert _native.get_stat("pm_halos") > 0
    o, energy, scale = oracle_core_diag(x, **kw)
    flips, worst = check_unbinding_band(g, o, energy, scale)
    print(f"fof_unbind_128 fp64={fp64}: {flips} flips, worst |E|/max|phi| = {worst:.2e}")
    check_ang_mom_consistent(g, x, kw["vp_list"], kw["mp_list"], wl["L"])


@pytest.mark.parametrize("fp64", [1, 0])
def test_unbind_nfw_2k(fp64):
    wl = bench.make_workload("unbind_nfw_2k", 0)
    x, kw = _kw(wl, True)
    with _native.options(unbind_fp64=fp64):
        g = P._fof_core(x, **kw)
    assert _native.get_stat("pm_halos") > 0
    assert max(a.shape[1] for a in x) > 32768
    o, energy, scale = oracle_core_diag(x, **kw)
    flips, worst = check_unbinding_band(g, o, energy, scale)
    print(f"unbind_nfw_2k fp64={fp64}: {flips} flips, worst |E|/max|phi| = {worst:.2e}")
    check_ang_mom_consistent(g, x, kw["vp_list"], None, wl["L"])
