"""Particle-mesh unbinding (candidates above 1000 members): the B200 solver
against the CPU oracle.

The oracle restates the reference PM algorithm with its own FP64 FFT in
place of FFTW3f, so PM parity is a tolerance, not bit equality:
  * first-pass potentials (C1 + C2): FP64 device path within 1e-5 of the
    oracle, FP32 product path within 1e-5 of the FP64 device path
    (relative to the halo's largest |phi|);
  * end-to-end membership: only particles whose oracle specific energy is
    within the energy band around zero (tests/helpers.py ENERGY_BAND times
    the halo's max |phi|) may be classified differently; halo counts and the
    ids of particles both keep are equal; each result's angular momentum
    matches its own members.
"""
import numpy as np
import pytest

import py_fof_b200 as P
from oracle import oracle as O
from py_fof_b200 import _native
from tests.helpers import check_ang_mom_consistent, check_unbinding_band, oracle_core_diag

pytestmark = pytest.mark.gpu

G = 1.0 / (6.0 * np.pi)
S15 = 15 * 0.67 * 512 / 300.0


def plummer(n, a, seed, rmax=None):
    rng = np.random.default_rng(seed)
    u = np.clip(rng.random(n), 1e-9, 1 - 1e-9)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    if rmax is not None:
        r = np.minimum(r, rmax)
    d = rng.standard_normal((3, n))
    d /= np.linalg.norm(d, axis=0)
    return r * d, r


def halo_q(n, a, seed, rmax):
    x, _ = plummer(n, a, seed, rmax)
    q = (x - x[:, :1]).astype(np.float32)
    w = np.random.default_rng(seed + 1).lognormal(-0.045, 0.3, n).astype(np.float32)
    return q, w


def oracle_phi(q, w):
    n = w.shape[0]
    xv = np.zeros((n, 6), np.float32)
    xv[:, :3] = q.T
    g, phi = O.first_potential(xv, w, np.arange(1, n + 1), softening=0.1, a_val=1.0, s15=S15)
    return g, phi


@pytest.mark.parametrize("n,a,rmax,expect_gid", [
    (1500, 0.3, 1.2, 1),     # 48 grid
    (1500, 0.4, 1.5, 2),     # 64 grid
    (4000, 3.0, 7.0, 3),     # 128 grid, coarse spacing
    (8000, 1.0, 5.0, 4),     # band 2, 256 grid
    (30000, 2.0, 7.0, 4),    # band 3, 256 grid
])
def test_first_pass_potential(n, a, rmax, expect_gid):
    q, w = halo_q(n, a, n, rmax)
    g_o, phi_o = oracle_phi(q, w)
    phi64, g64 = _native.halo_potential(q, w, fp64=True, s15=S15)
    phi32, g32 = _native.halo_potential(q, w, fp64=False, s15=S15)
    assert g_o == g64 == g32 == expect_gid
    if n == 30000:
        assert _native.get_stat("refined_regions") > 0
    scale = np.abs(phi_o).max()
    err64 = np.abs(phi64 - phi_o).max() / scale
    err32 = np.abs(phi32 - phi64).max() / scale
    assert err64 < 1e-5, err64
    assert err32 < 1e-5, err32
    # physics check: PM + C2 against the exact softened direct sum
    exact = O.direct_potential_f64(q.T, w, softening=0.1)
    assert np.abs(phi64 - exact).max() / np.abs(exact).max() < 3e-2


def _pm_halos(seed, sizes):
    rng = np.random.default_rng(seed)
    xs, vs, ms = [], [], []
    for k, n in enumerate(sizes):
        a = rng.uniform(0.6, 1.2)
        x, r = plummer(n, a, seed * 100 + k, rmax=5 * a)
        c = rng.uniform(50, 450, (3, 1))
        xs.append(c + x)
        m = rng.lognormal(-0.045, 0.3, n)
        sig = np.sqrt(G * n / (6.0 * np.sqrt(r * r + a * a)))
        v = rng.standard_normal((3, n)) * sig
        kk = rng.choice(n, n // 10, replace=False)
        v[:, kk] *= 4.0
        vs.append(v)
        ms.append(m)
    return xs, vs, ms


@pytest.mark.parametrize("fp64", [True, False])
def test_pm_unbinding_end_to_end(fp64):
    xs, vs, ms = _pm_halos(7, [1200, 2500, 4000, 9000, 1100, 600, 300])
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    with _native.options(unbind_fp64=int(fp64)):
        g = P._fof_core(xs, **kw)
    assert _native.get_stat("pm_halos") >= 3
    o, energy, scale = oracle_core_diag(xs, **kw)
    assert int(o[0].sum()) > 1000
    flips, worst = check_unbinding_band(g, o, energy, scale)
    print(f"pm fp64={fp64}: {flips} flips, worst |E|/max|phi| = {worst:.2e}")
    check_ang_mom_consistent(g, xs, vs, ms, 512.0)


@pytest.mark.parametrize("fp64", [True, False])
def test_large_halo_removal_loop(fp64):
    """A halo above the chunked-loop threshold (32768 members): the removal
    loop spread over the GPU against the oracle."""
    xs, vs, ms = _pm_halos(21, [40000, 3000, 1500])
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    with _native.options(unbind_fp64=int(fp64)):
        g = P._fof_core(xs, **kw)
    o, energy, scale = oracle_core_diag(xs, **kw)
    assert int(o[0].sum()) > 30000
    flips, worst = check_unbinding_band(g, o, energy, scale)
    print(f"large halo fp64={fp64}: {flips} flips, worst |E|/max|phi| = {worst:.2e}")
    check_ang_mom_consistent(g, xs, vs, ms, 512.0)


def test_chunked_loop_equals_block_loop():
    """Every PM halo through the chunked removal loop (threshold lowered)
    against the one-block loop: the same algorithm, centre sums in another
    order, so only particles inside the energy band may differ."""
    xs, vs, ms = _pm_halos(7, [1200, 2500, 4000, 9000, 1100, 600, 300])
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    with _native.options(unbind_fp64=1):
        a = P._fof_core(xs, **kw)
        with _native.options(unbind_big_np=1000):
            b = P._fof_core(xs, **kw)
    _, energy, scale = oracle_core_diag(xs, **kw)
    check_unbinding_band(a, b, energy, scale)
