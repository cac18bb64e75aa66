"""Brute-force friends-of-friends checker -- TEST INFRASTRUCTURE ONLY.

A second restatement of the reference's linking rule, written directly in
NumPy and independent of the C oracle (``oracle_fof.c``) and of the CUDA
library: every pair of a region is tested with the reference's exact
floating-point arithmetic, the accepted pairs are joined by
``scipy.sparse.csgraph.connected_components`` and the groups are numbered
the way the reference numbers them.  It is meant for small inputs (a few
thousand particles per region: the pair test is O(N^2)); tests and the
fixture generator ``tests/golden/make_periodic_golden.py`` use it.

What it restates (file:line in the reference project):

* unwrap about the region's first particle, ``x_rel = MODULO(x - x_anchor +
  L/2, L) - L/2`` in FP64 with gfortran's real MODULO
  (``fof_fortran.f90:521-523``), bounding box and periodic axes
  (``:525-533``);
* the cell geometry (``:535-570``) and each particle's cell
  ``i_d = min(N_d, max(1, floor((x_rel_d - origin_d)/size_d) + 1))``
  (``:579-585``) -- only used here to decide which pairs the reference's
  cell stencil visits and to order the groups;
* the pair set: the reference tests a pair iff its cells differ by at most
  one along every axis (wrapping on periodic axes); open regions use the
  13-half-neighbour stencil plus the in-cell triangle (``:625-657``),
  periodic regions the de-duplicated 26-neighbour set (``:717-755``).  Both
  visit every unordered pair of adjacent cells exactly once;
* the distance test on the FP32 stored coordinates ``x_crs =
  real(x_rel, 4)`` (``:599``): open regions square and sum in FP32 (x, y, z
  order) and compare in FP64 (``:636``); periodic regions use ``dist2_pbc``
  (``:483-491``): FP32 difference widened to FP64, ``L - dx`` beyond
  ``L/2``, FP64 squares summed x, y, z; a pair links iff ``r2 <= link**2``
  (``rp2`` in FP64, ``:518``);
* numbering: the DSU root of a group is its smallest CRS position
  (``atomic_dsu.c:25-39``, ``fof_fortran.f90:452-458``), CRS order is
  (cell, then ascending index inside a cell) (``:593-606``); candidates
  (size >= np_halo_min) are numbered by ascending root position
  (``:865-871``), regions in input order, regions below np_halo_min skipped
  (``fof_fortran.f90:164``).
"""
from __future__ import annotations

import math

import numpy as np


def fortran_modulo(a, p):
    """gfortran's real MODULO: fmod, then add p where the remainder is
    non-zero and its sign differs from p's."""
    r = np.fmod(a, p)
    fix = (r != 0.0) & ((r < 0.0) != (p < 0.0))
    return np.where(fix, r + p, r)


def cell_geometry(x_rel, L, link):
    """Per-axis (periodic, origin, N, size) of one region
    (fof_fortran.f90:525-570)."""
    n = x_rel.shape[1]
    lo = x_rel.min(axis=1)
    hi = x_rel.max(axis=1)
    rng = hi - lo
    periodic = [bool(rng[d] + 2.0 * link >= L) for d in range(3)]
    vol = max(float(rng[0]), link) * max(float(rng[1]), link) * max(float(rng[2]), link)

    def dims(L_mesh):
        out = []
        for d in range(3):
            if periodic[d]:
                N = max(1, min(int(L / link), int(L / L_mesh)))
                out.append((True, -0.5 * L, N, L / float(N)))
            else:
                N = max(1, int(math.ceil(float(rng[d]) / L_mesh)))
                out.append((False, float(lo[d]), N, L_mesh))
        return out

    L_mesh = max(link, (vol / float(max(1, n))) ** (1.0 / 3.0))
    g = dims(L_mesh)
    if float(g[0][2]) * float(g[1][2]) * float(g[2][2]) > float(max(262144, 4 * n)):
        L_mesh = max(link, (vol / float(max(1, n) * 2)) ** (1.0 / 3.0))
        g = dims(L_mesh)
    return g


def _cells(x_rel, geom):
    idx = []
    for d in range(3):
        _, origin, N, size = geom[d]
        i = np.floor((x_rel[d] - origin) / size).astype(np.int64) + 1
        idx.append(np.minimum(N, np.maximum(1, i)))
    return idx


def region_groups(x, L, link, np_min):
    """Groups of one region.  Returns a list of member arrays (local indices,
    ascending), in the reference's candidate order."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    x = np.asarray(x, dtype=np.float64)
    n = x.shape[1]
    half = 0.5 * L
    x_rel = fortran_modulo(x - x[:, :1] + half, L) - half
    geom = cell_geometry(x_rel, L, link)
    periodic_region = any(g[0] for g in geom)
    ci = _cells(x_rel, geom)
    icell = ci[0] + geom[0][2] * (ci[1] - 1) + geom[0][2] * geom[1][2] * (ci[2] - 1)
    xc = x_rel.astype(np.float32)
    rp2 = link * link

    rows, cols = [], []
    step = max(1, 4_000_000 // max(n, 1))
    for s in range(0, n, step):
        a = np.arange(s, min(n, s + step))
        # pairs (a, b) with b > a
        adj = np.ones((a.size, n), dtype=bool)
        for d in range(3):
            per, _, N, _ = geom[d]
            diff = ci[d][None, :] - ci[d][a, None]
            if per:
                diff = np.mod(diff, N)
                ok = (diff == 0) | (diff == 1) | (diff == N - 1)
            else:
                ok = np.abs(diff) <= 1
            adj &= ok
        adj &= np.arange(n)[None, :] > a[:, None]
        if periodic_region:
            r2 = np.zeros((a.size, n), dtype=np.float64)
            for d in range(3):
                dx = np.abs((xc[d][a, None] - xc[d][None, :]).astype(np.float64))
                dx = np.where(dx > half, L - dx, dx)
                r2 = r2 + dx * dx
        else:
            s32 = np.zeros((a.size, n), dtype=np.float32)
            for d in range(3):
                dx = xc[d][a, None] - xc[d][None, :]
                s32 = s32 + dx * dx
            r2 = s32.astype(np.float64)
        hit = adj & (r2 <= rp2)
        ia, ib = np.nonzero(hit)
        rows.append(a[ia])
        cols.append(ib)
    rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    g = coo_matrix((np.ones(rows.size, np.int8), (rows, cols)), shape=(n, n))
    _, label = connected_components(g, directed=False)
    # CRS position of each particle: cell, then index inside a cell
    crs = np.empty(n, np.int64)
    crs[np.lexsort((np.arange(n), icell))] = np.arange(n)
    groups = {}
    for p in range(n):
        groups.setdefault(int(label[p]), []).append(p)
    cands = [(int(crs[m].min()), np.asarray(m, np.int64)) for m in groups.values()
             if len(m) >= np_min]
    cands.sort(key=lambda t: t[0])
    return [m for _, m in cands]


def fof_brute(xp_list, L, link, np_min):
    """in_halo (int32 0/1) and halo_id (int32, reference numbering) of a
    list of (3, N_i) regions, or one (3, N) array."""
    if isinstance(xp_list, np.ndarray):
        xp_list = [xp_list]
    total = sum(x.shape[1] for x in xp_list)
    in_halo = np.zeros(total, np.int32)
    halo_id = np.zeros(total, np.int32)
    off, hid = 0, 0
    for x in xp_list:
        n = x.shape[1]
        if n >= np_min and n > 0:
            for m in region_groups(x, float(L), float(link), int(np_min)):
                hid += 1
                in_halo[off + m] = 1
                halo_id[off + m] = hid
        off += n
    return in_halo, halo_id
