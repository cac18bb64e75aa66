"""Unbinding parity: the B200 solvers against the CPU oracle.

* FP64 path (option unbind_fp64=1, the library default): the
  direct-summation removal loop reproduces the reference arithmetic, so
  in_halo and halo_id are bit-exact;
* FP32 product path (unbind_fp64=0): potentials carry FP32 rounding
  (compensated sums), so only a particle whose oracle specific energy lies
  within the energy band (tests/helpers.py ENERGY_BAND times its halo's
  max |phi|) may be classified differently; the halo count, the halo ids of
  particles both keep, and the angular momentum of each result's own
  members must agree.
"""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native
from tests.helpers import (angmom_close, check_ang_mom_consistent, check_unbinding_band,
                           oracle_core, oracle_core_diag)

pytestmark = pytest.mark.gpu

G = 1.0 / (6.0 * np.pi)


def clumps(seed, n_regions=60, nmin=20, nmax=1000, L=512.0, kick=0.1, masses=False):
    """Isolated Plummer clumps, one region each, virial velocities plus a
    kicked fraction, so every candidate takes the direct-summation path."""
    rng = np.random.default_rng(seed)
    xs, vs, ms = [], [], []
    for k in range(n_regions):
        n = int(rng.integers(nmin, nmax + 1))
        a = rng.uniform(0.3, 0.8)
        u = np.clip(rng.random(n), 1e-9, 1 - 1e-9)
        r = np.minimum(a / np.sqrt(u ** (-2.0 / 3.0) - 1.0), 4 * a)
        d = rng.standard_normal((3, n))
        d /= np.linalg.norm(d, axis=0)
        c = rng.uniform(20, L - 20, (3, 1))
        xs.append(c + r * d)
        sig = np.sqrt(G * n / (6.0 * np.sqrt(r * r + a * a)))
        v = rng.standard_normal((3, n)) * sig
        nk = int(kick * n)
        idx = rng.choice(n, nk, replace=False)
        v[:, idx] *= rng.uniform(2.0, 6.0, nk)
        vs.append(v + rng.standard_normal((3, 1)))
        ms.append(rng.lognormal(-0.045, 0.3, n) if masses else None)
    return xs, vs, (ms if masses else None)


@pytest.fixture
def fp64_path():
    with _native.options(unbind_fp64=1):
        yield


@pytest.mark.parametrize("seed,masses,hubble", [(1, False, False), (2, True, False), (3, True, True)])
def test_direct_fp64_bit_exact(fp64_path, seed, masses, hubble):
    xs, vs, ms = clumps(seed, masses=masses)
    kw = dict(vp_list=vs, L_Box=512.0, linking_length=0.3, np_halo_min=10, bound_check=True,
              return_ang_mom=True)
    if ms is not None:
        kw["mp_list"] = ms
    if hubble:
        kw["include_hubble_flow"] = True
        kw["z"] = 0.5
    g = P._fof_core(xs, **kw)
    o = oracle_core(xs, **kw)
    assert _native.get_stat("direct_halos") > 0
    assert o[1].max() > 0
    assert np.array_equal(g[0], o[0])
    assert np.array_equal(g[1], o[1])
    assert angmom_close(g[2], o[2], np.abs(o[2]).max() + 1.0)


def test_direct_fp32_product_path():
    xs, vs, ms = clumps(4, n_regions=80, masses=True)
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    with _native.options(unbind_fp64=0):
        g = P._fof_core(xs, **kw)
    o, energy, scale = oracle_core_diag(xs, **kw)
    assert int(o[0].sum()) > 1000
    flips, worst = check_unbinding_band(g, o, energy, scale)
    print(f"fp32 direct: {flips} flips, worst |E|/max|phi| = {worst:.2e}")
    check_ang_mom_consistent(g, xs, vs, ms, 512.0)
    check_ang_mom_consistent(o, xs, vs, ms, 512.0)


def test_direct_many_small_halos_in_box(fp64_path):
    """Candidates found by FoF in one periodic box, then unbound."""
    from py_fof_b200 import workloads as W
    d = W.plummer_box(32 ** 3, 32.0, 8, seed=5, with_velocities=True, lognormal_mass=0.3,
                      mmax=800)
    kw = dict(vp_list=d["vp"], mp_list=d["mp"], L_Box=32.0, linking_length=0.2, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    g = P._fof_core(d["xp"], **kw)
    o = oracle_core(d["xp"], **kw)
    assert np.array_equal(g[1], o[1])
    assert angmom_close(g[2], o[2], np.abs(o[2]).max() + 1.0)


def test_too_few_and_all_unbound(fp64_path):
    """Halos that lose too many members end with status TOO_FEW and no output."""
    xs, vs, _ = clumps(6, n_regions=20, kick=0.0)
    vs = [v * 50.0 for v in vs]
    kw = dict(vp_list=vs, L_Box=512.0, linking_length=0.3, np_halo_min=10, bound_check=True)
    g = P._fof_core(xs, **kw)
    o = oracle_core(xs, **kw)
    assert np.array_equal(g[1], o[1])


def test_per_halo_baseline_matches_batched():
    """The plain per-halo FP64 baseline (one halo per launch sequence) and the
    batched FP64 path compute each halo with the same kernels and the same
    summation order (the mesh deposit is deterministic), so they agree bit
    for bit."""
    from tests.test_pm_gpu import _pm_halos
    xs, vs, ms = clumps(8, n_regions=30, masses=True)
    xp, vp, mp = _pm_halos(11, [1300, 2200])
    xs, vs, ms = xs + xp, vs + vp, ms + mp
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    with _native.options(unbind_fp64=1):
        a = P._fof_core(xs, **kw)
        with _native.options(unbind_per_halo=1):
            b = P._fof_core(xs, **kw)
            assert _native.get_stat("pm_halos") >= 1
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert angmom_close(a[2], b[2], np.abs(a[2]).max() + 1.0)


def test_fp32_runs_reproduce():
    """Two runs of the FP32 product path on the same input give the same
    bits: no result depends on the order of atomic additions."""
    from tests.test_pm_gpu import _pm_halos
    xs, vs, ms = clumps(9, n_regions=20, masses=True)
    xp, vp, mp = _pm_halos(12, [1500, 4000, 9000])
    xs, vs, ms = xs + xp, vs + vp, ms + mp
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    with _native.options(unbind_fp64=0):
        a = P._fof_core(xs, **kw)
        b = P._fof_core(xs, **kw)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
