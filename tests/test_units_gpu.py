"""Unit conversion on the device (pyfof_run_units): the public calls pass the
caller's arrays and the conversion to code units; the library divides and
multiplies on the device.  Results must equal the oracle fed with the
host-converted arrays (py_fof/__init__.py:266-326): FoF bit-exact,
angular momenta to summation-order rounding, unbinding within the
particle-mesh tolerance."""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native, workloads as W
from tests.helpers import check_unbinding_band, oracle_core_diag, angmom_close, oracle_core

pytestmark = pytest.mark.gpu


def _physical_box(seed):
    d = W.plummer_box(32 ** 3, 32.0, 8, seed=seed, with_velocities=True)
    rng = np.random.default_rng(seed)
    mp = rng.lognormal(np.log(4e10), 0.3, d["xp"].shape[1])
    # positions in Mpc/h in a 32 Mpc/h box, velocities in km/s, masses in Msun/h
    return d["xp"], 120.0 * d["vp"], mp


@pytest.mark.parametrize("mass", ["array", "scalar", "n_sim"])
def test_physical_fof_matches_host_conversion(mass):
    xp, vp, mp = _physical_box(1)
    kw = dict(vp_list=vp, L_Box=32.0, linking_length=0.1, np_halo_min=10, units="physical",
              z=0.5, return_ang_mom=True, n_sim=64 ** 3)
    if mass == "array":
        kw["mp_list"] = mp
    elif mass == "scalar":
        kw["mp_list"] = 3.3e10
    call = P._prepare(xp, check_masses=False, device_units=True, **kw)
    assert call.units is not None and call.units[0] == 0.5
    g = P._fof_core(xp, **kw)
    o = oracle_core(xp, **kw)
    assert o[1].max() > 0
    assert np.array_equal(g[0], o[0]) and np.array_equal(g[1], o[1])
    assert angmom_close(g[2], o[2], np.abs(o[2]).max() + 1.0)


def test_scalar_mass_cube_units():
    d = W.plummer_box(32 ** 3, 32.0, 8, seed=2, with_velocities=True)
    kw = dict(vp_list=d["vp"], L_Box=32.0, linking_length=0.2, np_halo_min=10, mp_list=2.5,
              return_ang_mom=True)
    assert P._prepare(d["xp"], device_units=True, **kw).mp is None  # travels as a constant
    g = P._fof_core(d["xp"], **kw)
    o = oracle_core(d["xp"], **kw)
    assert np.array_equal(g[1], o[1])
    assert angmom_close(g[2], o[2], np.abs(o[2]).max() + 1.0)


def test_physical_unbinding_within_tolerance():
    xs, vs = W.nfw_halos(12, seed=5, sizes=[40, 90, 300, 700, 1500, 2600, 30, 60, 150, 400, 900, 5000])
    # the generator's grid units -> Mpc/h and km/s of a 256 Mpc/h box sampled
    # by 512^3 particles (dx = 0.5 Mpc/h)
    dx, v_scale = 0.5, 512.0 / (150.0 * np.sqrt(0.3) * 256.0)
    xs_phys = [x * dx for x in xs]
    vs_phys = [v / v_scale for v in vs]
    kw = dict(vp_list=vs_phys, L_Box=256.0, linking_length=0.2 * dx, np_halo_min=10, bound_check=True,
              units="physical", softening=0.1 * dx, n_sim=512 ** 3, ng_global=512.0)
    assert P._prepare(xs_phys, device_units=True, **kw).units[0] == dx
    g = P._fof_core(xs_phys, **kw)
    o, energy, scale = oracle_core_diag(xs_phys, **kw)
    assert int(o[0].sum()) > 1000
    check_unbinding_band(g, o, energy, scale)


def test_invalid_raw_mass_rejected_before_conversion():
    xp, vp, mp = _physical_box(3)
    mp[1234] = -1.0
    kw = dict(vp_list=vp, L_Box=32.0, linking_length=0.1, units="physical", mp_list=mp)
    with pytest.raises(ValueError, match="positive and finite"):
        P.fof(xp, **kw)
    # the context stays usable
    mp[1234] = 1e10
    assert P.fof(xp, **kw).shape == (xp.shape[1],)


def test_units_entry_point_with_slot():
    xp, vp, mp = _physical_box(4)
    kw = dict(vp_list=vp, L_Box=32.0, linking_length=0.1, units="physical", mp_list=mp, n_sim=64 ** 3)
    call = P._prepare(xp, check_masses=False, device_units=True, **kw)
    slot = _native.slot_create(0, 1 << 30)
    try:
        a = _native.run(call.xp, call.vp, call.mp, call.np_halo, call.nhalo, call.L_Box, call.link,
                        call.np_halo_min, call.bound_check, call.verbose, call.softening, call.a_val,
                        call.b_val, call.s_15_val, call.n_threads, call.total_np, slot=slot,
                        units=call.units)
    finally:
        _native.slot_destroy(slot)
    h = call.on_host()
    b = _native.run(h.xp, h.vp, h.mp, h.np_halo, h.nhalo, h.L_Box, h.link, h.np_halo_min, h.bound_check,
                    h.verbose, h.softening, h.a_val, h.b_val, h.s_15_val, h.n_threads, h.total_np)
    assert a[3] == 0 and b[3] == 0
    assert np.array_equal(a[1], b[1])
    assert angmom_close(a[2], b[2], np.abs(b[2]).max() + 1.0)
