"""Generate tests/golden/periodic_fof.npz: small friends-of-friends inputs
whose partitions are decided by the brute-force checker
(``oracle/brute_force.py``), independent of the C oracle and of the CUDA
library.

    python tests/golden/make_periodic_golden.py

The cases exercise the reference's periodic branch (``dist2_pbc``,
``fof_fortran.f90:483-491``, wrapped 26-neighbour cells ``:717-755``) where
no test of the reference itself pins a result: boxes of 1, 2 and 3 cells per
axis, clumps straddling faces and corners, pairs placed on either side of the
linking length in FP32 (inside the box and across the periodic boundary),
coordinates given outside [0, L), a region periodic along one axis only,
a list of regions mixing open and periodic ones, and very dense clumps in
link-sized cells (one across a corner of the box).  Every input is seeded.
The fixture stores, per case, the positions, the region sizes, L, the
linking length, np_halo_min and the expected in_halo / halo_id.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.brute_force import cell_geometry, fof_brute, fortran_modulo  # noqa: E402

OUT = os.path.join(HERE, "periodic_fof.npz")


def clumps(rng, L, centres, counts, scale):
    pts = []
    for c, k in zip(centres, counts):
        pts.append(np.asarray(c, float)[:, None] + rng.normal(0.0, scale, (3, k)))
    return np.hstack(pts)


def wrap_some(rng, x, L, frac=0.1):
    """Give a fraction of the coordinates outside [0, L) (shifted by +-L):
    the reference unwraps them with MODULO before anything else."""
    x = np.mod(x, L)
    m = rng.random(x.shape) < frac
    s = rng.choice([-1.0, 1.0], x.shape)
    return np.where(m, x + s * L, x)


def boundary_pair_offsets(x1, L, link):
    """FP32 coordinates x2 along one axis such that the pair (x1, x2) sits
    on either side of the linking length under dist2_pbc: returns (the
    largest separation that links, the smallest that does not)."""
    half = 0.5 * L
    rp2 = link * link
    a = np.float32(x1)
    target = np.float32(x1 + link)
    cands = [target]
    up = down = target
    for _ in range(8):
        up = np.nextafter(up, np.float32(np.inf))
        down = np.nextafter(down, np.float32(-np.inf))
        cands += [up, down]
    res = []
    for b in sorted(set(float(c) for c in cands)):
        dx = abs(float(np.float32(a) - np.float32(b)))
        if dx > half:
            dx = L - dx
        res.append((b, dx * dx <= rp2))
    inside = max(b for b, ok in res if ok)
    outside = min(b for b, ok in res if not ok)
    return inside, outside


def case_boundary_pairs(rng):
    """Pairs a linking length apart to the last FP32 ulp.  The x_rel of a
    single-region input is relative to the first particle, so the first
    particle sits at 0 and every pair is built in x_rel coordinates."""
    L, link = 8.0, 0.2
    pts = [np.zeros(3)]
    # background keeps the region periodic along every axis
    pts += list(rng.uniform(-L / 2, L / 2, (40, 3)))
    for k in range(12):
        base = rng.uniform(-L / 2 + 1.6, L / 2 - 1.6, 3)
        axis = k % 3
        across = k >= 6
        x1 = float(np.float32(base[axis]))
        if across:
            x1 = float(np.float32(L / 2 - 0.05))  # partner lands across +L/2
        inside, outside = boundary_pair_offsets(x1, L, link)
        for x2, shift in ((inside, 0.0), (outside, 1.5)):
            p = base.copy()
            p[(axis + 1) % 3] += shift
            p1 = p.copy()
            p1[axis] = x1
            p2 = p.copy()
            p2[axis] = x2
            if across:
                p2[axis] = x2 - L  # the same point, expressed inside the box
            pts += [p1, p2]
    xr = np.array(pts).T
    # x_rel of these positions is themselves (anchor at 0): check that the
    # unwrap keeps them, so the FP32 pair spacing is the one built above
    half = 0.5 * L
    back = fortran_modulo(xr - xr[:, :1] + half, L) - half
    assert np.array_equal(back.astype(np.float32), xr.astype(np.float32))
    return dict(xp=xr, np_halo=[xr.shape[1]], L=L, link=link, np_min=2)


def main():
    cases = {}
    rng = np.random.default_rng(20261204)

    # clumps across faces and corners in a box of many cells
    L = 10.0
    cen = [(0.1, 5, 5), (9.95, 9.9, 0.05), (5, 0.02, 5), (3, 3, 3), (7, 2, 9.9)]
    x = np.hstack([rng.uniform(0, L, (3, 2100)), clumps(rng, L, cen, [300, 250, 150, 120, 80], 0.25)])
    cases["pbc_clumps"] = dict(xp=wrap_some(rng, x, L), np_halo=[x.shape[1]], L=L, link=0.2, np_min=5)

    # denser box, longer link
    L = 12.0
    cen = rng.uniform(0, L, (12, 3))
    x = np.hstack([rng.uniform(0, L, (3, 3000)), clumps(rng, L, cen, [170] * 12, 0.35)])
    cases["pbc_dense"] = dict(xp=wrap_some(rng, x, L), np_halo=[x.shape[1]], L=L, link=0.35, np_min=10)

    # tight clumps on a lattice of spacing L/2 in a unit box: the linking
    # length sets 1, 2 or 3 cells per (periodic) axis; the clump at the
    # origin straddles every face
    lattice = [(0, 0, 0), (0.5, 0.5, 0.5), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5),
               (0.5, 0, 0), (0, 0.5, 0), (0, 0, 0.5)]
    for name, link, cen in (("pbc_1cell", 0.55, lattice[:2]), ("pbc_2cell", 0.4, lattice[2:5] + lattice[:1]),
                            ("pbc_3cell", 0.3, lattice)):
        L = 1.0
        x = clumps(rng, L, cen, [8] * len(cen), 0.03)
        x = np.hstack([x, rng.uniform(0, L, (3, 3))])
        cases[name] = dict(xp=wrap_some(rng, x, L, 0.2), np_halo=[x.shape[1]], L=L, link=link,
                           np_min=2)

    cases["pbc_boundary_pairs"] = case_boundary_pairs(rng)

    # a filament: periodic along z only, open along x and y
    L = 20.0
    z = rng.uniform(0, L, 500)
    xy = rng.normal(0.0, 0.4, (2, 500)) + 7.0
    x = np.hstack([np.vstack([xy, z]), clumps(rng, L, [(7, 7, 0.02), (7.2, 6.9, 10)], [60, 60], 0.1)])
    cases["pbc_partial"] = dict(xp=wrap_some(rng, x, L), np_halo=[x.shape[1]], L=L, link=0.2, np_min=5)

    # a list of regions: open clumps, a periodic box, one below np_halo_min
    L = 64.0
    regs = [clumps(rng, L, [(30, 30, 30)], [800], 0.3),
            np.hstack([rng.uniform(0, 6.0, (3, 900)) + 0.0,
                       clumps(rng, L, [(0.05, 3, 3)], [200], 0.2)]),
            clumps(rng, L, [(10, 50, 5)], [4], 0.05),
            np.hstack([rng.uniform(0, L, (3, 1500)),
                       clumps(rng, L, [(63.95, 0.02, 32), (20, 63.9, 63.99)], [150, 100], 0.2)]),
            clumps(rng, L, [(60, 2, 40), (61, 3, 41)], [300, 300], 0.4)]
    # the second region spans [0,6) only, so it is open unless wrapped:
    # put half its particles near L so it straddles the x face
    regs[1][0, :450] = np.mod(regs[1][0, :450] - 3.0, L)
    cases["list_mixed"] = dict(xp=np.hstack(regs), np_halo=[r.shape[1] for r in regs], L=L,
                               link=0.2, np_min=10)

    # very dense clumps in a periodic box of link-sized cells (one across a
    # corner): cells of hundreds of particles, linked by merge sub-cells
    L = 2.0
    cen = [(0.02, 1.98, 0.01), (1.0, 1.0, 1.0), (0.5, 1.4, 0.6)]
    x = np.hstack([rng.uniform(0, L, (3, 600)), clumps(rng, L, cen, [1600, 1200, 500], 0.05)])
    cases["pbc_very_dense"] = dict(xp=wrap_some(rng, x, L), np_halo=[x.shape[1]], L=L, link=0.2, np_min=5)

    out = {}
    for name, c in cases.items():
        xp = np.ascontiguousarray(c["xp"], dtype=np.float64)
        nph = np.asarray(c["np_halo"], np.int32)
        offs = np.concatenate([[0], np.cumsum(nph)])
        regions = [xp[:, offs[i]:offs[i + 1]] for i in range(len(nph))]
        in_halo, halo_id = fof_brute(regions, c["L"], c["link"], c["np_min"])
        half = 0.5 * c["L"]
        ncells = []
        for r in regions:
            g = cell_geometry(fortran_modulo(r - r[:, :1] + half, c["L"]) - half, c["L"], c["link"])
            ncells.append([g[d][2] for d in range(3)] + [int(g[d][0]) for d in range(3)])
        print(f"{name:20s} N={xp.shape[1]:5d} groups={int(halo_id.max()):4d} "
              f"members={int(in_halo.sum()):5d} cells/periodic={ncells}")
        out[f"{name}__xp"] = xp
        out[f"{name}__np_halo"] = nph
        out[f"{name}__params"] = np.array([c["L"], c["link"], c["np_min"]], np.float64)
        out[f"{name}__in_halo"] = in_halo
        out[f"{name}__halo_id"] = halo_id
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
