"""Periodic-branch parity pinned by the brute-force checker.

``tests/golden/periodic_fof.npz`` holds small inputs whose partitions were
decided by ``oracle/brute_force.py`` -- every pair tested in the reference's
arithmetic (``dist2_pbc``, ``fof_fortran.f90:483-491``; open regions
``:636``), groups numbered by their smallest CRS position -- independently
of the C oracle and of the CUDA library.  Both must reproduce them exactly:
in_halo and halo_id bit for bit.
"""
import numpy as np
import pytest

from tests.helpers import GOLDEN, oracle_core

CASES = ["pbc_clumps", "pbc_dense", "pbc_1cell", "pbc_2cell", "pbc_3cell", "pbc_boundary_pairs",
         "pbc_partial", "list_mixed", "pbc_very_dense"]


def _case(name):
    d = np.load(f"{GOLDEN}/periodic_fof.npz")
    xp = d[f"{name}__xp"]
    nph = d[f"{name}__np_halo"]
    L, link, np_min = d[f"{name}__params"]
    offs = np.concatenate([[0], np.cumsum(nph)])
    regions = [np.ascontiguousarray(xp[:, offs[i]:offs[i + 1]]) for i in range(len(nph))]
    inp = regions if len(regions) > 1 else regions[0]
    kw = dict(L_Box=float(L), linking_length=float(link), np_halo_min=int(np_min))
    return inp, kw, d[f"{name}__in_halo"], d[f"{name}__halo_id"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_brute_force(name):
    inp, kw, in_halo, halo_id = _case(name)
    o = oracle_core(inp, **kw)
    assert np.array_equal(np.asarray(o[0], np.int32), in_halo)
    assert np.array_equal(o[1], halo_id)


def test_fixture_regenerates():
    """The checker reproduces the committed answers (a few cases)."""
    from oracle.brute_force import fof_brute
    for name in ("pbc_3cell", "pbc_boundary_pairs", "list_mixed"):
        inp, kw, in_halo, halo_id = _case(name)
        regions = inp if isinstance(inp, list) else [inp]
        ih, hid = fof_brute(regions, kw["L_Box"], kw["linking_length"], kw["np_halo_min"])
        assert np.array_equal(ih, in_halo) and np.array_equal(hid, halo_id)


def test_boundary_pairs_split_at_link():
    """The boundary case holds pairs that link and pairs one FP32 ulp
    farther that do not: both outcomes must be present."""
    _, _, in_halo, halo_id = _case("pbc_boundary_pairs")
    assert halo_id.max() >= 12
    assert (in_halo == 0).sum() >= 24


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_brute_force(name):
    import py_fof_b200 as P
    inp, kw, in_halo, halo_id = _case(name)
    from py_fof_b200 import _native
    g = P._fof_core(inp, **kw)
    if name == "pbc_very_dense":
        assert _native.get_stat("vd_cells") > 0  # linked by merge sub-cells
    assert np.array_equal(np.asarray(g[0], np.int32), in_halo)
    assert np.array_equal(g[1], halo_id)
