"""FoF parity: the B200 path (py_fof_b200 -> libpyfof_b200.so) against the
CPU oracle on seeded inputs.  The partition, in_halo and halo_id (reference
numbering) must be bit-exact; angular momenta agree to summation-order
rounding."""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import _native, workloads as W
from tests.helpers import angmom_close, canonical, oracle_core

pytestmark = pytest.mark.gpu


def _both(xp_list, **kw):
    g = P._fof_core(xp_list, **kw)
    o = oracle_core(xp_list, **kw)
    return g, o


def _assert_same(g, o, scale=1.0):
    assert np.array_equal(g[0], o[0]), "in_halo differs"
    assert np.array_equal(g[1], o[1]), "halo_id differs"
    assert angmom_close(g[2], o[2], scale), f"ang_mom {g[2]} vs {o[2]}"


def test_library_loads_native():
    L = _native.load()
    assert L.pyfof_version() == _native.ABI_VERSION
    assert L.pyfof_init(0) == 0


@pytest.mark.parametrize("seed", [0, 1])
def test_config1_recipe_small(seed):
    d = W.plummer_box(32 ** 3, 32.0, 8, seed=seed, with_velocities=True)
    g, o = _both(d["xp"], vp_list=d["vp"], L_Box=32.0, linking_length=0.2, np_halo_min=10,
                 return_ang_mom=True)
    assert o[1].max() > 0
    _assert_same(g, o, scale=np.abs(o[2]).max() + 1.0)


def test_config1_full_size():
    d = W.config1(seed=3)
    g, o = _both(d["xp"], L_Box=64.0, linking_length=0.2, np_halo_min=10)
    assert o[1].max() > 10
    _assert_same(g, o)


def test_open_region_clustered():
    rng = np.random.default_rng(7)
    xp = np.concatenate([rng.normal(200.0, 3.0, (3, 20000)),
                         rng.uniform(150.0, 250.0, (3, 5000))], axis=1)
    vp = rng.normal(0.0, 1.0, xp.shape)
    g, o = _both(xp, vp_list=vp, L_Box=512.0, linking_length=0.4, np_halo_min=5,
                 return_ang_mom=True)
    assert o[1].max() > 0
    _assert_same(g, o, scale=np.abs(o[2]).max() + 1.0)


def test_multi_region_mixed():
    rng = np.random.default_rng(11)
    xs, vs = [], []
    for k, n in enumerate([500, 3, 0, 4000, 12, 2500, 9]):
        c = rng.uniform(0, 100, (3, 1))
        xs.append(c + rng.normal(0, 1.5, (3, n)))
        vs.append(rng.normal(0, 0.3, (3, n)))
    g, o = _both(xs, vp_list=vs, L_Box=100.0, linking_length=0.35, np_halo_min=10,
                 return_ang_mom=True)
    _assert_same(g, o, scale=np.abs(o[2]).max() + 1.0)


@pytest.mark.parametrize("L,link", [(0.3, 0.2), (0.5, 0.2), (1.0, 0.3), (2.0, 0.3)])
def test_small_periodic_boxes(L, link):
    """Boxes with 1, 2 and 3 cells per axis exercise the neighbour dedup."""
    rng = np.random.default_rng(int(L * 100))
    xp = rng.uniform(0, L, (3, 400))
    g, o = _both(xp, L_Box=L, linking_length=link, np_halo_min=3)
    _assert_same(g, o)


@pytest.mark.parametrize("L,link,n", [(3.0, 0.5, 40), (2.0, 0.6, 12), (1.2, 0.5, 20), (1.5, 0.45, 30),
                                      (5.0, 0.6, 200), (7.0, 1.1, 150)])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_sparse_small_periodic_boxes(L, link, n, seed):
    """Few particles per cell in boxes of 2 to 6 cells per axis: the row
    kernel's wrapped ranges, shifted boxes and skipped rows."""
    rng = np.random.default_rng(seed + int(10 * L))
    xp = rng.uniform(0, L, (3, n))
    g, o = _both(xp, L_Box=L, linking_length=link, np_halo_min=2)
    _assert_same(g, o)


def test_sparse_rows_with_dense_cells():
    """Sparse rows interleaved with dense cells, in a periodic box and in an
    open region: pairs between sparse and dense cells from both sides."""
    rng = np.random.default_rng(11)
    for L, open_region in ((24.0, False), (1000.0, True)):
        lo = 0.0 if not open_region else 400.0
        span = L if not open_region else 24.0
        back = rng.uniform(lo, lo + span, (3, int(2.5 * span ** 3)))
        cents = rng.uniform(lo, lo + span, (3, 40))
        clumps = np.concatenate([c[:, None] + rng.normal(0, 0.15, (3, 60)) for c in cents.T], axis=1)
        xp = np.concatenate([back, clumps], axis=1)
        if not open_region:
            xp = np.mod(xp, L)
        g, o = _both(xp, L_Box=L, linking_length=0.2, np_halo_min=5)
        assert o[1].max() > 10
        _assert_same(g, o)


@pytest.mark.parametrize("clump", [200, 3000, 12000])
def test_cell_order_paths(clump):
    """The stable cell order by per-cell sorts (cells up to 8192 particles,
    small ones by insertion, larger ones by a block sort) and by the radix
    sort (a fuller cell): the same partition and numbering as the oracle."""
    rng = np.random.default_rng(clump)
    back = rng.uniform(0, 40.0, (3, 60000))
    cents = rng.uniform(0, 40.0, (3, 6))
    clumps = [c[:, None] + rng.normal(0, 0.12, (3, clump)) for c in cents.T]
    xp = np.mod(np.concatenate([back] + clumps, axis=1), 40.0)
    o = oracle_core(xp, L_Box=40.0, linking_length=0.2, np_halo_min=10)
    for mode in (1, 2, 0):
        _native.set_option("cell_order", mode)
        try:
            g = P._fof_core(xp, L_Box=40.0, linking_length=0.2, np_halo_min=10)
        finally:
            _native.set_option("cell_order", 0)
        m = _native.get_stat("max_cell")
        assert (m > 8192) == (clump == 12000) and m > 32
        # per-cell sorts only where asked for and every cell fits a block
        assert _native.get_stat("cell_sorts") == (1 if (mode == 1 and m <= 8192) else 0)
        _assert_same(g, o)


def test_partially_periodic_filament():
    rng = np.random.default_rng(5)
    n = 6000
    xp = np.stack([rng.uniform(0, 50.0, n), 25 + rng.normal(0, 0.4, n),
                   25 + rng.normal(0, 0.4, n)])
    g, o = _both(xp, L_Box=50.0, linking_length=0.25, np_halo_min=10)
    assert o[1].max() > 0
    _assert_same(g, o)


def test_degenerate_positions():
    xp = np.zeros((3, 50))
    xp[0, 25:] = 3.0
    g, o = _both(xp, L_Box=10.0, linking_length=0.2, np_halo_min=10)
    _assert_same(g, o)
    assert g[1].max() == 2


def test_link_length_boundary():
    """Pairs placed at the linking length: FP32 rounding decides them."""
    rng = np.random.default_rng(9)
    base = rng.uniform(10, 90, (3, 300))
    d = rng.standard_normal((3, 300))
    d /= np.linalg.norm(d, axis=0)
    xp = np.concatenate([base, base + 0.2 * d], axis=1)
    for L in (100.0, 1e4):
        g, o = _both(xp, L_Box=L, linking_length=0.2, np_halo_min=2)
        _assert_same(g, o)


@pytest.mark.parametrize("npmin", [1, 2, 1000000])
def test_np_halo_min_extremes(npmin):
    rng = np.random.default_rng(2)
    xp = rng.uniform(0, 20, (3, 3000))
    g, o = _both(xp, L_Box=20.0, linking_length=0.5, np_halo_min=npmin)
    _assert_same(g, o)


@pytest.mark.parametrize("L", [30.0, 60.0])
def test_dense_clumps_across_boundary(L):
    """Clumps much denser than one particle per cell, some straddling the
    periodic faces and corners, exercise the sub-cell index of dense cells."""
    rng = np.random.default_rng(int(L))
    parts = [rng.uniform(0, L, (3, 20000))]
    for c in ([0.0, 0.0, 0.0], [L / 2, 0.05, L - 0.05], [L / 3, L / 3, L / 3]):
        parts.append(np.array(c)[:, None] + rng.normal(0, 0.25, (3, 4000)))
    xp = np.mod(np.concatenate(parts, axis=1), L)
    g, o = _both(xp, L_Box=L, linking_length=0.2, np_halo_min=10)
    assert _native.get_stat("dense_cells") > 0
    assert o[1].max() >= 3
    _assert_same(g, o)


def test_dense_clumps_open_region():
    rng = np.random.default_rng(21)
    parts = [rng.uniform(100, 140, (3, 30000))]
    for k in range(5):
        parts.append(rng.uniform(100, 140, (3, 1)) + rng.normal(0, 0.3, (3, 3000)))
    xp = np.concatenate(parts, axis=1)
    g, o = _both(xp, L_Box=1000.0, linking_length=0.25, np_halo_min=10)
    assert _native.get_stat("dense_cells") > 0
    _assert_same(g, o)


def test_fortran_order_input():
    d = W.plummer_box(16 ** 3, 16.0, 2, seed=4)
    xf = np.asfortranarray(d["xp"])
    a = P._fof_core(xf, L_Box=16.0, linking_length=0.2, np_halo_min=5)
    b = P._fof_core(d["xp"], L_Box=16.0, linking_length=0.2, np_halo_min=5)
    assert np.array_equal(a[1], b[1])


def test_empty_and_errors():
    r = P._fof_core(np.zeros((3, 0)))
    assert r[0].shape == (0,) and r[2].shape == (3, 1)
    bad = np.array([[np.nan, 0.0], [0.0, 0.0], [0.0, 0.0]])
    with pytest.raises(ValueError):
        P.fof(bad, L_Box=10.0, np_halo_min=1)
    # a region below np_halo_min is skipped without being read, as in the reference
    assert not P.fof(bad, L_Box=10.0, np_halo_min=10).any()


def test_device_entry_point_matches_host():
    torch = pytest.importorskip("torch")
    d = W.plummer_box(24 ** 3, 24.0, 4, seed=8)
    ref = P._fof_core(d["xp"], L_Box=24.0, linking_length=0.2, np_halo_min=10)
    x = torch.from_numpy(d["xp"]).cuda()
    n = d["xp"].shape[1]
    ih = torch.zeros(n, dtype=torch.int32, device="cuda")
    hid = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    am, ierr = _native.run_device(x.data_ptr(), 0, 0, _native.LAYOUT_SOA, [n], 1, n, 24.0, 0.2,
                                  10, 0, 0, 0.1, 1.0, 0.0, 1.0, 0, ih.data_ptr(), hid.data_ptr())
    assert ierr == 0
    assert np.array_equal(hid.cpu().numpy(), ref[1])
    assert np.array_equal(ih.cpu().numpy().astype(bool), ref[0])


def test_canonical_partition_matches():
    d = W.plummer_box(20 ** 3, 20.0, 3, seed=12)
    g, o = _both(d["xp"], L_Box=20.0, linking_length=0.25, np_halo_min=2)
    assert np.array_equal(canonical(g[1]), canonical(o[1]))


@pytest.mark.parametrize("bad_mass", [0.0, -1.0, np.nan, np.inf])
@pytest.mark.parametrize("bound", [False, True])
def test_invalid_masses_rejected_on_device(bad_mass, bound):
    """The mass check (py_fof/__init__.py:259-260) runs on the device for
    the native call and raises the reference's ValueError; the oracle path
    keeps the host check, with the same message."""
    d = W.plummer_box(12 ** 3, 12.0, 2, seed=21, with_velocities=True, lognormal_mass=0.3)
    mp = d["mp"].copy()
    mp[777] = bad_mass
    kw = dict(vp_list=d["vp"], mp_list=mp, L_Box=12.0, linking_length=0.2, np_halo_min=10,
              bound_check=bound, ng_global=512.0)
    with pytest.raises(ValueError, match="positive and finite"):
        P.fof(d["xp"], **kw)
    with pytest.raises(ValueError, match="positive and finite"):
        oracle_core(d["xp"], **kw)
    # the library stays usable and a valid call afterwards is unaffected
    kw["mp_list"] = d["mp"]
    assert np.array_equal(P._fof_core(d["xp"], **kw)[1], oracle_core(d["xp"], **kw)[1])


@pytest.mark.parametrize("seed", [1, 2])
def test_lognormal_field_partition(seed):
    """The large-FoF configuration's recipe at reduced size (lognormal field,
    sigma_G = 1.5, P(k) ~ k^-2, np_halo_min 20): dense clumps next to voids,
    groups that span many cells; bit-exact with the oracle."""
    x = W.lognormal_box(96 ** 3, 96.0, 48, seed=seed)
    kw = dict(L_Box=96.0, linking_length=0.2, np_halo_min=20)
    g, o = _both(x, **kw)
    assert o[1].max() > 20
    assert np.array_equal(g[0], o[0])
    assert np.array_equal(g[1], o[1])
    # the cell order by per-cell sorts (the path of the largest boxes)
    _native.set_option("cell_order", 1)
    try:
        g1 = P._fof_core(x, **kw)
    finally:
        _native.set_option("cell_order", 0)
    assert _native.get_stat("cell_sorts") == 1
    assert np.array_equal(g1[0], o[0]) and np.array_equal(g1[1], o[1])


@pytest.mark.parametrize("seed", [3, 4])
def test_very_dense_periodic_clumps(seed):
    """Clumps dense enough that link-sized cells hold hundreds of particles,
    one across a corner of the periodic box: those cells are linked by merge
    sub-cells (all pairs inside one are linked) and sub-cell pairs; the
    partition must still be the reference's, bit for bit."""
    rng = np.random.default_rng(seed)
    L = 6.0
    cen = np.array([[0.03, 5.98, 0.02], [3.0, 3.0, 3.0], [1.5, 4.2, 2.0], [5.0, 1.0, 4.5]])
    x = [rng.uniform(0, L, (3, 20000))]
    for c, k, sc in zip(cen, [4000, 3000, 2000, 1500], [0.08, 0.1, 0.06, 0.15]):
        x.append(c[:, None] + rng.normal(0.0, sc, (3, k)))
    xp = np.mod(np.hstack(x), L)
    kw = dict(L_Box=L, linking_length=0.2, np_halo_min=5)
    g = P._fof_core(xp, **kw)
    assert _native.get_stat("vd_cells") > 0
    o = oracle_core(xp, **kw)
    assert np.array_equal(g[0], o[0])
    assert np.array_equal(g[1], o[1])


@pytest.mark.parametrize("n", [1, 3, 4, 5, 4099, 20 ** 3 + 3])
def test_mask_entry_point_matches_halo_ids(n):
    """pyfof_run_mask (what fof() calls) returns halo_id > 0 as bytes, for
    sizes that leave 0-3 particles past the last group of four."""
    rng = np.random.default_rng(n)
    L = 20.0
    xp = np.hstack([rng.uniform(0, L, (3, n // 2)),
                    rng.normal(L / 2, 0.3, (3, n - n // 2))])
    full = P._fof_core(xp, L_Box=L, linking_length=0.2, np_halo_min=2)
    in_halo, hid, am, ierr = _native.run(xp, None, None, [n], 1, L, 0.2, 2, 0, 0, 0.1, 1.0, 0.0,
                                         17.152, 0, n, mask_only=True)
    assert ierr == 0 and hid is None and in_halo.dtype == np.bool_
    assert np.array_equal(in_halo, full[1] > 0)
    assert np.array_equal(P.fof(xp, L_Box=L, linking_length=0.2, np_halo_min=2), full[0])


def test_mask_public_fof_with_unbinding_and_regions():
    """fof() through the mask entry point against _fof_core: isolated bound
    clumps as a list of regions (some below np_halo_min), with unbinding."""
    from tests.test_unbind_gpu import clumps
    xs, vs, ms = clumps(7, n_regions=12, nmin=5, nmax=600, masses=True)
    xs.insert(3, xs[3][:, :4].copy())  # a region below np_halo_min
    vs.insert(3, vs[3][:, :4].copy())
    ms.insert(3, ms[3][:4].copy())
    kw = dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.3, np_halo_min=10,
              bound_check=True, return_ang_mom=True)
    core = P._fof_core(xs, **kw)
    ih, am = P.fof(xs, **kw)
    assert core[1].max() > 0 and min(x.shape[1] for x in xs) < 10
    assert ih.dtype == np.bool_
    # ang_mom sums members with atomics: equal to rounding
    assert np.array_equal(ih, core[0]) and angmom_close(am, core[2], np.abs(core[2]).max() + 1.0)
    # one periodic box, positions only
    d = W.plummer_box(24 ** 3, 24.0, 4, seed=21)
    core = P._fof_core(d["xp"], L_Box=24.0, linking_length=0.2, np_halo_min=10)
    assert core[1].max() > 0
    assert np.array_equal(P.fof(d["xp"], L_Box=24.0, linking_length=0.2, np_halo_min=10), core[0])


def test_mask_zeroed_on_failure():
    xp = np.zeros((3, 6))
    xp[0, 2] = np.nan
    in_halo, _, am, ierr = _native.run(xp, None, None, [6], 1, 10.0, 0.2, 1, 0, 0, 0.1, 1.0, 0.0,
                                       17.152, 0, 6, mask_only=True)
    assert ierr == 4 and not in_halo.any() and not am.any()


def test_list_inputs_through_page_locked_staging():
    """Lists of regions (with velocity and mass lists) are concatenated into
    the thread's page-locked staging; it is reused and grown from call to
    call, and every call equals the oracle."""
    rng = np.random.default_rng(33)
    for nreg, per in ((5, 50), (40, 300), (3, 20), (60, 700)):
        xs = [rng.normal(rng.uniform(5, 59, (3, 1)), 0.15, (3, int(rng.integers(per // 2, per + 1))))
              for _ in range(nreg)]
        vs = [rng.normal(0, 1, x.shape) for x in xs]
        ms = [rng.lognormal(0, 0.2, x.shape[1]) for x in xs]
        kw = dict(vp_list=vs, mp_list=ms, L_Box=64.0, linking_length=0.2, np_halo_min=5,
                  return_ang_mom=True)
        ih, am = P.fof(xs, **kw)
        info = P.fof_with_info(xs, **kw)
        o = oracle_core(xs, **kw)
        assert np.array_equal(ih, o[0]) and np.array_equal(info["in_halo"], o[0])
        assert angmom_close(am, o[2], np.abs(o[2]).max() + 1.0)
    assert _native.thread_staging().cap > 0
