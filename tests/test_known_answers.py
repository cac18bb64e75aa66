"""The reference's known-answer tests (test_fof.py:653-1169), run against the
CPU oracle (pins the oracle) and against the B200 product path.

Inputs come from tests/golden/*.npz, produced by the reference's own
generator (tests/golden/make_golden.py); the expected answers are the ones
the reference tests assert.
"""
import numpy as np
import pytest

import py_fof_b200 as P
from tests.helpers import LINK, L_BOX, NP_MIN, golden, oracle_fof, oracle_fof_with_info

BACKENDS = [
    pytest.param("oracle", id="oracle"),
    pytest.param("gpu", id="gpu", marks=pytest.mark.gpu),
]


def _api(backend):
    if backend == "oracle":
        return oracle_fof, oracle_fof_with_info
    return P.fof, P.fof_with_info


@pytest.mark.parametrize("backend", BACKENDS)
def test_predictable_halo(backend):
    fof, _ = _api(backend)
    g = golden("predictable_halo")
    in_halo, am = fof(g["xp"], L_Box=L_BOX, linking_length=LINK, np_halo_min=NP_MIN,
                      return_ang_mom=True)
    assert np.allclose(am, 0.0)
    assert np.array_equal(in_halo, g["expected"])


@pytest.mark.parametrize("backend", BACKENDS)
def test_predictable_halo_with_velocity(backend):
    fof, _ = _api(backend)
    g = golden("predictable_halo_velocity")
    plain = fof(g["xp"], L_Box=L_BOX, linking_length=LINK, np_halo_min=NP_MIN)
    bound, am = fof(g["xp"], vp_list=g["vp"], L_Box=L_BOX, linking_length=LINK,
                    np_halo_min=NP_MIN, bound_check=True, return_ang_mom=True)
    assert am.shape == (3, 1)
    unbound = plain & ~bound
    assert unbound[g["high_v"]].all()
    assert bound.sum() == int(g["expected_bound"])


@pytest.mark.parametrize("backend", BACKENDS)
def test_multiple_predictable_halos(backend):
    fof, _ = _api(backend)
    g = golden("multiple_halos")
    in_halo = fof([g["xp0"], g["xp1"], g["xp2"]], L_Box=L_BOX, linking_length=LINK,
                  np_halo_min=NP_MIN)
    assert np.array_equal(in_halo, g["expected"])


@pytest.mark.parametrize("backend", BACKENDS)
def test_multiple_predictable_halos_with_velocity(backend):
    fof, _ = _api(backend)
    g = golden("multiple_halos_velocity")
    xs = [g["xp0"], g["xp1"], g["xp2"]]
    vs = [g["vp0"], g["vp1"], g["vp2"]]
    plain = fof(xs, L_Box=L_BOX, linking_length=LINK, np_halo_min=NP_MIN)
    bound = fof(xs, vp_list=vs, L_Box=L_BOX, linking_length=LINK, np_halo_min=NP_MIN,
                bound_check=True)
    unbound = plain & ~bound
    assert unbound[g["high_v"]].all()
    assert bound.sum() == int(g["expected_bound"])


@pytest.mark.parametrize("backend", BACKENDS)
def test_new_features(backend):
    fof, fof_with_info = _api(backend)
    g = golden("new_features")
    xs = [g["xp0"], g["xp1"], g["xp2"]]
    vs = [g["vp0"], g["vp1"], g["vp2"]]
    kw = dict(L_Box=L_BOX, linking_length=LINK, np_halo_min=NP_MIN)
    # [1] fof_with_info agrees with fof
    info = fof_with_info(xs, vp_list=vs, bound_check=True, return_ang_mom=True, **kw)
    in_halo, am = fof(xs, vp_list=vs, bound_check=True, return_ang_mom=True, **kw)
    assert np.array_equal(info["in_halo"], in_halo)
    assert info["nhalo_found"] == int(g["nhalo_expected"])
    assert len(info["halo_indices"]) == int(g["nhalo_expected"])
    assert np.sum(info["np_per_halo"]) == np.sum(info["in_halo"])
    allidx = np.concatenate(info["halo_indices"])
    assert len(allidx) == len(np.unique(allidx))
    assert np.all(info["in_halo"][allidx])
    assert np.allclose(info["ang_mom"], am)
    # [2] n_threads does not change the result; > 256 raises
    base = fof(xs, vp_list=vs, bound_check=True, n_threads=1, return_ang_mom=True, **kw)
    for nt in (2, 4, None):
        r = fof(xs, vp_list=vs, bound_check=True, n_threads=nt, return_ang_mom=True, **kw)
        assert np.array_equal(r[0], base[0])
        assert np.allclose(r[1], base[1], atol=1e-12)
    with pytest.raises(ValueError):
        fof(xs, n_threads=300)
    # [3] scalar mass == array mass; a heavy centre binds at least as much
    total = sum(x.shape[1] for x in xs)
    a = fof(xs, vp_list=vs, bound_check=True, mp_list=1.0, **kw)
    b = fof(xs, vp_list=vs, bound_check=True, mp_list=np.ones(total), **kw)
    assert np.array_equal(a, b)
    xs1, vs1 = g["xp_single"], g["vp_single"]
    light = fof(xs1, vp_list=vs1, bound_check=True, mp_list=1.0, **kw)
    heavy_m = np.ones(100)
    heavy_m[0] = 200.0
    heavy = fof(xs1, vp_list=vs1, bound_check=True, mp_list=heavy_m, **kw)
    assert heavy.sum() >= light.sum()
    # [4] physical units: softening required; cube == physical
    with pytest.raises(ValueError):
        fof(xs1, vp_list=vs1, units="physical", bound_check=True)
    ng, box_mpc = 512.0, 300.0
    dx = box_mpc / ng
    v_factor = 150.0 * np.sqrt(0.3) * box_mpc / (1.0 * ng)
    m_grid = 0.3 * 2.77536627e11 * (box_mpc ** 3) / (ng ** 3)
    inh_c, am_c = fof(xs1, vp_list=vs1, L_Box=ng, linking_length=LINK, np_halo_min=NP_MIN,
                      bound_check=True, mp_list=heavy_m, softening=0.1, units="cube",
                      return_ang_mom=True)
    inh_p, am_p = fof(xs1 * dx, vp_list=vs1 * v_factor, L_Box=box_mpc,
                      linking_length=LINK * dx, np_halo_min=NP_MIN, bound_check=True,
                      mp_list=heavy_m * m_grid, softening=0.1 * dx, units="physical",
                      return_ang_mom=True)
    assert np.array_equal(inh_c, inh_p)
    assert np.allclose(am_c * (m_grid * dx * v_factor), am_p, rtol=1e-5)
    hf = fof(xs1 * dx, vp_list=vs1 * v_factor, L_Box=box_mpc, linking_length=LINK * dx,
             np_halo_min=NP_MIN, bound_check=True, mp_list=heavy_m * m_grid,
             softening=0.1 * dx, units="physical", include_hubble_flow=True)
    assert isinstance(hf, np.ndarray)


@pytest.mark.parametrize("backend", BACKENDS)
def test_span_limit(backend):
    fof, _ = _api(backend)
    g = golden("overspan")
    with pytest.raises(ValueError, match="exceeds"):
        fof(g["xp"], vp_list=g["vp"], L_Box=L_BOX, linking_length=LINK, np_halo_min=NP_MIN,
            bound_check=True, box=300.0, h0=0.67)
