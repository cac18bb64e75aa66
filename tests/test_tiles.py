"""The tile table: launch shapes that must never change a result.

CPU: the table file format, validation of keys and values through the
C-ABI (no device work).  GPU: one input with direct-summation halos of every
size bucket and particle-mesh halos of every grid gives the same in_halo
and halo_id bits under every candidate value of every entry."""
import json

import numpy as np
import pytest

from py_fof_b200 import _native, autotune


def test_set_get_and_validation():
    old = _native.get_tile("direct_threads", 0)
    try:
        for v in (32, 64, 128, 256):
            _native.set_tile("direct_threads", 0, v)
            assert _native.get_tile("direct_threads", 0) == v
        for bad in (("direct_threads", 0, 48), ("direct_threads", 6, 64), ("pm_batch", 100, 4),
                    ("conv_waves", 64, 0), ("conv_waves", 64, 65), ("no_such", 0, 1)):
            with pytest.raises(ValueError):
                _native.set_tile(*bad)
    finally:
        _native.set_tile("direct_threads", 0, old)


def test_table_file_roundtrip(tmp_path):
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"device": "x", "direct_threads": {"0": 32, "5": 256},
                             "pm_batch": {"256": 16}, "conv_waves": {"48": 2}}))
    ent = _native.read_tile_table(str(p))
    assert ("direct_threads", 0, 32) in ent and ("pm_batch", 256, 16) in ent
    keep = [(k, i, _native.get_tile(k, i)) for k, i, _ in ent]
    try:
        assert _native.apply_tile_table(str(p)) == str(p)
        assert _native.get_tile("conv_waves", 48) == 2
    finally:
        for k, i, v in keep:
            _native.set_tile(k, i, v)
    p.write_text(json.dumps({"direct_threads": {"0": 48}}))
    with pytest.raises(ValueError):
        _native.apply_tile_table(str(p))


def test_committed_table_is_valid():
    import os
    if os.path.exists(_native.TILE_TABLE):
        for key, idx, val in _native.read_tile_table(_native.TILE_TABLE):
            old = _native.get_tile(key, idx)
            _native.set_tile(key, idx, val)
            _native.set_tile(key, idx, old)


@pytest.mark.gpu
def test_results_identical_under_every_entry():
    import py_fof_b200 as P
    rng = np.random.default_rng(5)
    sizes = [int(rng.integers(lo, hi + 1)) for lo, hi in autotune.BUCKETS for _ in range(6)]
    xs, vs = autotune.plummer_clumps(9, sizes)
    for n in autotune.GRIDS:
        x, v = autotune.pm_halos_for_grid(n, 100 + n, 2 if n < 256 else 1)
        xs += x
        vs += v
    kw = dict(vp_list=vs, L_Box=512.0, linking_length=0.3, np_halo_min=10, bound_check=True)
    for fp64 in (1, 0):
        with _native.options(unbind_fp64=fp64):
            ref = P._fof_core(xs, **kw)
            assert _native.get_stat("pm_halos") >= 4
            entries = ([("direct_threads", b, t) for b in range(6) for t in autotune.THREADS] +
                       [("pm_batch", n, c) for n in autotune.GRIDS for c in (1, 3)] +
                       [("conv_waves", n, c) for n in autotune.GRIDS for c in (1, 16)])
            for e in entries:
                with _native.tiles(e):
                    g = P._fof_core(xs, **kw)
                assert np.array_equal(g[0], ref[0]), e
                assert np.array_equal(g[1], ref[1]), e
