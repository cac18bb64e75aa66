"""The allocation-free potential entry point against the pool-allocating one.

pyfof_halo_potential_direct_static serves callers that must not allocate
device memory while they run (a framework whose allocator already owns the
device, or a step loop that cannot afford an allocation failure): its
scratch is a static device array of the library.  Both entry points run the
same direct-summation kernel, so their potentials must agree exactly; two
calls in a row with different sizes (the first at the 1000-member limit)
check that no state leaks between calls through the shared array, and the
device's free memory is unchanged across calls.  This file is collected
last on purpose.
"""
import numpy as np
import pytest

from py_fof_b200 import _native

pytestmark = pytest.mark.gpu


def _halo(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, 0.5, (3, n))
    q = (x - x[:, :1]).astype(np.float32)
    w = rng.lognormal(-0.045, 0.3, n).astype(np.float32)
    return q, w


@pytest.mark.parametrize("fp64", [True, False])
def test_static_matches_pool_entry_point_twice(fp64):
    assert _native.load().pyfof_init(0) == 0
    for n, seed in ((1000, 1), (250, 2)):
        q, w = _halo(n, seed)
        ref, meth = _native.halo_potential(q, w, fp64=fp64)
        assert meth == 0
        got, ierr = _native.halo_potential_direct_static(q, w, fp64=fp64)
        assert ierr == 0, _native.last_error()
        np.testing.assert_array_equal(got, ref)


def test_static_allocates_nothing():
    """After a first call (per-device set-up, kernel loading), further calls
    leave the device's free memory exactly as it was."""
    import torch
    assert _native.load().pyfof_init(0) == 0
    q, w = _halo(600, 4)
    _, ierr = _native.halo_potential_direct_static(q, w)
    assert ierr == 0, _native.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for n, seed in ((1000, 5), (37, 6), (999, 7)):
        q, w = _halo(n, seed)
        _, ierr = _native.halo_potential_direct_static(q, w, fp64=n % 2 == 1)
        assert ierr == 0, _native.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)


def test_static_rejects_oversized_candidates():
    q, w = _halo(1001, 3)
    _, ierr = _native.halo_potential_direct_static(q, w)
    assert ierr == 1
    assert "exceed" in _native.last_error()
