"""CPU-side checks of the native boundary: the C-ABI library loads without a
GPU and exports every symbol include/pyfof_b200.h declares; the Python
wrapper validates arguments like the reference."""
import os
import re

import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "pyfof_b200.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pyfof_\w+)\s*\(", src)))


def test_header_matches_binding():
    assert sorted(_native.EXPORTED) == _declared()


def test_library_exports_all_symbols():
    L = _native.load()
    for name in _declared():
        assert hasattr(L, name), name
    assert L.pyfof_version() == _native.ABI_VERSION


def test_validation_errors():
    xp = np.zeros((3, 5))
    with pytest.raises(ValueError):
        P.fof(xp, units="bogus")
    with pytest.raises(ValueError):
        P.fof(xp, n_threads=300)
    with pytest.raises(ValueError):
        P.fof(np.zeros((2, 5)))
    with pytest.raises(ValueError):
        P.fof(xp, bound_check=True)
    with pytest.raises(ValueError):
        P.fof(xp, vp_list=[xp, xp])
    with pytest.raises(ValueError):
        P.fof(xp, mp_list=-1.0)
    with pytest.raises(ValueError):
        P.fof(xp, z=-1.0)
    with pytest.raises(ValueError):
        P.fof(xp, vp_list=xp, bound_check=True, units="physical")
    with pytest.raises(ValueError):
        P.fof(xp, vp_list=xp, bound_check=True, units="physical", softening=0.1)


def test_empty_input_returns_zeros():
    r = P._fof_core([np.zeros((3, 0)), np.zeros((3, 0))])
    assert r[0].shape == (0,) and r[1].shape == (0,) and r[2].shape == (3, 2)


def test_prepare_units():
    xp = np.random.default_rng(0).uniform(0, 10, (3, 20))
    c = P._prepare(xp, units="physical", L_Box=300.0, linking_length=0.1)
    assert c.L_Box == 512.0
    assert np.allclose(c.xp, xp / (300.0 / 512.0))
    c = P._prepare(xp, ng_global=256.0, L_Box=128.0)
    assert np.isclose(c.s_15_val, 15 * 0.67 * 256.0 / 300.0)


@pytest.mark.parametrize("mass", ["array", "scalar", "n_sim", "none", "per_region"])
@pytest.mark.parametrize("units", ["physical", "cube"])
def test_device_units_carry_the_host_conversion(mass, units):
    """_prepare(device_units=True) leaves the arrays in the caller's units and
    carries the conversion; applying it (FofCall.on_host, the operations the
    device performs) gives the host-converted call bit for bit."""
    rng = np.random.default_rng(4)
    xs = [rng.uniform(0, 300.0, (3, 40)), rng.uniform(0, 300.0, (3, 25))]
    vs = [rng.normal(0, 300.0, (3, 40)), rng.normal(0, 300.0, (3, 25))]
    kw = dict(vp_list=vs, L_Box=300.0, linking_length=0.3, units=units, z=0.7, softening=0.02,
              bound_check=True, include_hubble_flow=True)
    if mass == "array":
        kw["mp_list"] = rng.uniform(1e9, 1e11, 65)
    elif mass == "scalar":
        kw["mp_list"] = 3.7e10
    elif mass == "n_sim":
        kw["n_sim"] = 256 ** 3
    elif mass == "per_region":
        kw["mp_list"] = [2e10, 5e9]
    elif units == "physical":
        kw["n_sim"] = 200 ** 3
    host = P._prepare(xs, **kw)
    dev = P._prepare(xs, device_units=True, **kw)
    if units == "physical":
        assert dev.units is not None and dev.units[0] != 1.0
        assert np.array_equal(dev.xp, np.hstack(xs))  # unconverted
    conv = dev.on_host()
    assert conv.units is None
    assert conv.xp.dtype == host.xp.dtype and np.array_equal(conv.xp, host.xp)
    # vp/mp may be absent on one side where the other holds zeros / ones
    for f in ("L_Box", "link", "softening", "a_val", "b_val", "s_15_val", "ang_mom_scale"):
        assert getattr(conv, f) == getattr(host, f), f
    assert all(x.dtype == y.dtype and np.array_equal(x, y) for x, y in zip(dev.dense(), host.dense()))


def test_options_validated():
    """Options are plain settings of the library (no device work): accepted
    values stick, others are refused with the library's message."""
    from py_fof_b200 import _native
    _native.set_option("cell_order", 1)
    _native.set_option("cell_order", 0)
    with pytest.raises(ValueError, match="cell_order"):
        _native.set_option("cell_order", 3)
    with pytest.raises(ValueError, match="unknown option"):
        _native.set_option("no_such_option", 1)


def test_catalogue_from_ids():
    hid = np.array([0, 2, 1, 2, 0, 1, 3], np.int32)
    res = P.catalogue_from_ids(hid > 0, hid)
    assert res["nhalo_found"] == 3
    assert [list(h) for h in res["halo_indices"]] == [[2, 5], [1, 3], [6]]
    assert list(res["np_per_halo"]) == [2, 2, 1]


class _HostStaging:
    """Stand-in for _native.Staging with ordinary memory: the same reserve /
    take contract (views into one buffer, reset by reserve)."""

    def __init__(self):
        self.buf = np.zeros(0, np.uint8)
        self.used = 0
        self.reserved = []

    def reserve(self, nbytes):
        self.reserved.append(nbytes)
        self.used = 0
        if nbytes > self.buf.size:
            self.buf = np.zeros(nbytes, np.uint8)
        return True

    def take(self, shape):
        n = int(np.prod(shape))
        off = (self.used + 255) // 256 * 256
        assert off + 8 * n <= self.buf.size
        self.used = off + 8 * n
        return self.buf[off:off + 8 * n].view(np.float64).reshape(shape)


def test_list_inputs_concatenated_into_staging():
    """Lists of regions (positions, velocities, masses) land in the staging
    buffer with the values np.hstack gives; single arrays are not copied."""
    rng = np.random.default_rng(5)
    xs = [rng.normal(size=(3, int(k))) for k in rng.integers(1, 400, 25)]
    vs = [rng.normal(size=x.shape) for x in xs]
    ms = [rng.uniform(0.5, 2.0, x.shape[1]) for x in xs]
    kw = dict(vp_list=vs, mp_list=ms, L_Box=50.0, bound_check=True, softening=0.1,
              check_masses=False, device_units=True)
    plain = P._prepare(xs, **kw)
    st = _HostStaging()
    staged = P._prepare(xs, staging=st, **kw)
    n = sum(x.shape[1] for x in xs)
    assert st.reserved and st.reserved[-1] >= 56 * n
    for a, b in ((plain.xp, staged.xp), (plain.vp, staged.vp), (plain.mp, staged.mp)):
        assert np.array_equal(a, b)
    for arr in (staged.xp, staged.vp, staged.mp):
        assert np.shares_memory(arr, st.buf)
    # one array: used as it is
    one = P._prepare(xs[0], L_Box=50.0, staging=_HostStaging(), device_units=True)
    assert one.xp is xs[0] or np.shares_memory(one.xp, xs[0])


def test_staging_unavailable_falls_back():
    class _NoStaging(_HostStaging):
        def reserve(self, nbytes):
            return False
    xs = [np.ones((3, 4)), np.zeros((3, 6))]
    c = P._prepare(xs, L_Box=10.0, staging=_NoStaging(), device_units=True)
    assert np.array_equal(c.xp, np.hstack(xs))
