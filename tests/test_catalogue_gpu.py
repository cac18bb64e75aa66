"""The fof_with_info catalogue built on the device (stable radix sort of the
particle indices by halo id, pyfof_run_catalogue) against the catalogue the
host derives from the same call's halo ids and against the oracle: halo
count, member counts and member lists must be identical."""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native, workloads as W
from tests.helpers import oracle_fof_with_info

pytestmark = pytest.mark.gpu


def _same_catalogue(a, b):
    assert a['nhalo_found'] == b['nhalo_found']
    assert np.array_equal(a['in_halo'], b['in_halo'])
    assert np.array_equal(a['np_per_halo'], b['np_per_halo'])
    assert len(a['halo_indices']) == len(b['halo_indices'])
    for x, y in zip(a['halo_indices'], b['halo_indices']):
        assert x.dtype == y.dtype and np.array_equal(x, y)
    assert np.array_equal(a['bound_status'], b['bound_status'])


def _device_and_host(xp_list, **kw):
    """Both catalogues of ONE native call: the device's and the one the host
    derives from that call's halo ids."""
    call = P._prepare(xp_list, check_masses=False, device_units=True, **kw)
    ih, hid, am, ierr, members, offsets = _native.run_catalogue(
        call.xp, call.vp, call.mp, call.np_halo, call.nhalo, call.L_Box, call.link, call.np_halo_min,
        call.bound_check, call.verbose, call.softening, call.a_val, call.b_val, call.s_15_val,
        call.n_threads, call.total_np, ng_val=call.ng_val, ng_global_val=call.ng_global_val,
        units=call.units)
    assert ierr == 0
    assert offsets[0] == 0 and np.all(np.diff(offsets) > 0) and offsets[-1] == members.size
    host = P.catalogue_from_ids(ih, hid)
    dev = {'in_halo': ih, 'nhalo_found': len(offsets) - 1, 'np_per_halo': np.diff(offsets),
           'halo_indices': np.split(members.astype(np.int64), offsets[1:-1]) if len(offsets) > 1 else [],
           'bound_status': np.zeros(len(offsets) - 1, dtype=np.int32)}
    return dev, host


def test_fof_only_matches_oracle():
    d = W.plummer_box(32 ** 3, 32.0, 8, seed=5, with_velocities=True)
    kw = dict(vp_list=d["vp"], L_Box=32.0, linking_length=0.2, np_halo_min=10, return_ang_mom=True)
    dev = P.fof_with_info(d["xp"], **kw)
    assert dev['nhalo_found'] > 0
    _same_catalogue(dev, oracle_fof_with_info(d["xp"], **kw))
    assert dev['ang_mom'].shape == (3, 1)
    _same_catalogue(*_device_and_host(d["xp"], **kw))


def test_bound_check_matches_host_catalogue():
    xs, vs = W.nfw_halos(8, seed=11, sizes=[300, 700, 1500, 2500, 40000, 6000, 25, 90])
    kw = dict(vp_list=vs, L_Box=512.0, linking_length=0.2, np_halo_min=20, bound_check=True)
    dev, host = _device_and_host(xs, **kw)
    assert dev['nhalo_found'] >= 6
    _same_catalogue(dev, host)
    # the public call returns the same structure
    pub = P.fof_with_info(xs, **kw)
    assert abs(pub['nhalo_found'] - dev['nhalo_found']) <= 1


def test_multi_region_list():
    rng = np.random.default_rng(3)
    xs = [np.concatenate([rng.normal(c, 1.5, (3, 4000)), rng.uniform(c - 20, c + 20, (3, 1000))], axis=1)
          for c in (50.0, 120.0, 300.0, 410.0)]
    kw = dict(L_Box=512.0, linking_length=0.3, np_halo_min=8)
    dev = P.fof_with_info(xs, **kw)
    assert dev['nhalo_found'] >= 4
    _same_catalogue(dev, oracle_fof_with_info(xs, **kw))


def test_no_halo_and_empty_inputs():
    rng = np.random.default_rng(1)
    xp = rng.uniform(0.0, 512.0, (3, 5000))  # mean spacing ~30, link 0.2: no groups of 10
    kw = dict(L_Box=512.0, linking_length=0.2, np_halo_min=10)
    dev = P.fof_with_info(xp, **kw)
    assert dev['nhalo_found'] == 0 and dev['halo_indices'] == [] and dev['np_per_halo'].size == 0
    _same_catalogue(dev, oracle_fof_with_info(xp, **kw))
    empty = P.fof_with_info(np.zeros((3, 0)), **kw)
    assert empty['nhalo_found'] == 0


def test_single_particle_halos():
    # np_halo_min = 1 makes every particle a halo: the largest id range the
    # offsets buffer has to hold
    rng = np.random.default_rng(2)
    xp = rng.uniform(0.0, 512.0, (3, 20000))
    kw = dict(L_Box=512.0, linking_length=0.2, np_halo_min=1)
    dev = P.fof_with_info(xp, **kw)
    assert dev['nhalo_found'] > 19000
    _same_catalogue(dev, oracle_fof_with_info(xp, **kw))
