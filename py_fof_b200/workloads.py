"""Seeded synthetic particle sets for benchmarks and tests.

No public dataset is involved: the benchmark configurations are described by
their recipe (particle count, box, clustering model), and these generators
produce float64 (3,N) C-order arrays with those shapes and distributions.

* ``plummer_box``: a periodic box with a uniform background plus Plummer
  spheres whose member counts follow dN/dM ~ M^-1.9, renormalised to a given
  halo fraction (the 64^3 / 256^3 FoF configurations).  Halo centres sit on
  a jittered lattice so neighbouring halos do not merge into groups wider
  than the unbinding span limit.
* ``nfw_halos``: a list of isolated NFW spheres (one region per halo) with
  power-law sizes, virial velocities and a kicked unbound fraction (the
  batched-unbinding configuration).
"""
from __future__ import annotations

import numpy as np

G_CODE = 1.0 / (6.0 * np.pi)   # a/(6 pi) at z = 0 (bound_fortran.f90:2616)


def _power_law_counts(rng, n_halos, total, mmin, mmax, slope=-1.9, floor=20):
    if total < n_halos * floor:
        raise ValueError(f"{total} halo particles cannot fill {n_halos} halos of at least {floor}")
    e = slope + 1.0
    u = rng.random(n_halos)
    m = (mmin ** e + u * (mmax ** e - mmin ** e)) ** (1.0 / e)
    c = np.floor(m / m.sum() * total).astype(np.int64)
    c = np.maximum(c, floor)
    diff = int(total - c.sum())
    idx = rng.permutation(n_halos)
    k = 0
    while diff != 0:
        j = idx[k % n_halos]
        step = 1 if diff > 0 else -1
        if c[j] + step >= floor:
            c[j] += step
            diff -= step
        k += 1
    return c


def plummer_box(n_total, L, n_halos, seed=0, a=1.5, halo_frac=0.3, mmin=20, mmax=5000,
                with_velocities=False, lognormal_mass=None, kick_frac=0.1, bulk_sigma=3.0,
                bg_sigma=1.0, shuffle=True):
    """Uniform background + Plummer halos in a periodic box of side L.

    Returns dict(xp, vp or None, mp or None, halo_of (member halo or -1)).
    """
    rng = np.random.default_rng(seed)
    n_h = int(round(halo_frac * n_total))
    n_bg = n_total - n_h
    counts = _power_law_counts(rng, n_halos, n_h, mmin, mmax)
    side = int(np.ceil(n_halos ** (1.0 / 3.0)))
    cells = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side),
                                 indexing="ij"), -1).reshape(-1, 3)[:n_halos]
    spacing = L / side
    centres = (cells + 0.5 + 0.25 * (rng.random((n_halos, 3)) - 0.5)) * spacing
    xs = [rng.random((3, n_bg)) * L]
    vs = [rng.standard_normal((3, n_bg)) * bg_sigma] if with_velocities else None
    owner = [np.full(n_bg, -1, np.int64)]
    for h in range(n_halos):
        m = int(counts[h])
        u = rng.random(m)
        u = np.clip(u, 1e-12, 1 - 1e-9)
        r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        d = rng.standard_normal((3, m))
        d /= np.linalg.norm(d, axis=0)
        xs.append(centres[h][:, None] + r * d)
        owner.append(np.full(m, h, np.int64))
        if with_velocities:
            sig = np.sqrt(G_CODE * m / (6.0 * np.sqrt(r * r + a * a)))
            v = rng.standard_normal((3, m)) * sig + rng.standard_normal((3, 1)) * bulk_sigma
            nk = int(kick_frac * m)
            if nk:
                k = rng.choice(m, nk, replace=False)
                kd = rng.standard_normal((3, nk))
                kd /= np.linalg.norm(kd, axis=0)
                v[:, k] += 3.0 * sig[k] * kd
            vs.append(v)
    xp = np.mod(np.concatenate(xs, axis=1), L)
    owner = np.concatenate(owner)
    vp = np.concatenate(vs, axis=1) if with_velocities else None
    mp = None
    if lognormal_mass is not None:
        s = float(lognormal_mass)
        mp = rng.lognormal(mean=-0.5 * s * s, sigma=s, size=n_total)
    if shuffle:
        p = rng.permutation(n_total)
        xp = xp[:, p]
        owner = owner[p]
        if vp is not None:
            vp = vp[:, p]
        if mp is not None:
            mp = mp[p]
    return dict(xp=np.ascontiguousarray(xp), vp=None if vp is None else np.ascontiguousarray(vp),
                mp=mp, halo_of=owner)


def config1(seed=0):
    """64^3 particles, L=64, 64 Plummer halos (FoF only)."""
    return plummer_box(64 ** 3, 64.0, 64, seed=seed)


def config2(seed=0, n_side=256):
    """n_side^3 particles in L=n_side with 4096 (scaled) Plummer halos,
    lognormal masses and velocities (FoF + unbinding)."""
    n_halos = max(1, int(round(4096 * (n_side / 256.0) ** 3)))
    return plummer_box(n_side ** 3, float(n_side), n_halos, seed=seed, with_velocities=True,
                       lognormal_mass=0.3)


def nfw_halos(n_halos, seed=0, mmin=20, mmax=2_000_000, s15=17.152, link=0.2, kick_frac=0.1,
              mean_density=None, sizes=None):
    """List of isolated NFW spheres (one region each) for batched unbinding.

    The virial radius is set by a fixed mean density inside R_vir chosen so
    that the largest halo spans at most 0.9 * s15 (R_vir <= 0.45 s15).
    Member counts follow dN/dM ~ M^-1.9 on [mmin, mmax] unless `sizes`
    gives them.  Returns (xp_list, vp_list).
    """
    rng = np.random.default_rng(seed)
    e = -0.9
    u = rng.random(n_halos)
    if sizes is None:
        sizes = np.floor((mmin ** e + u * (mmax ** e - mmin ** e)) ** (1.0 / e)).astype(np.int64)
    else:
        sizes = np.asarray(sizes, np.int64)
    rv_max = 0.45 * s15
    if mean_density is None:
        mean_density = mmax / (4.0 / 3.0 * np.pi * rv_max ** 3)
    xs, vs = [], []
    for m in sizes:
        m = int(m)
        rv = (m / (4.0 / 3.0 * np.pi * mean_density)) ** (1.0 / 3.0)
        c = rng.uniform(5.0, 15.0)
        rs = rv / c
        mu = lambda x: np.log1p(x) - x / (1.0 + x)
        # inverse CDF by bisection on x = r/rs in [0, c]
        target = rng.random(m) * mu(c)
        lo = np.zeros(m)
        hi = np.full(m, c)
        for _ in range(50):
            mid = 0.5 * (lo + hi)
            f = mu(mid) < target
            lo = np.where(f, mid, lo)
            hi = np.where(f, hi, mid)
        r = 0.5 * (lo + hi) * rs
        d = rng.standard_normal((3, m))
        d /= np.linalg.norm(d, axis=0)
        centre = rng.uniform(100.0, 400.0, 3)
        xs.append(centre[:, None] + r * d)
        menc = m * mu(r / rs) / mu(c)
        sig = np.sqrt(G_CODE * np.maximum(menc, 1.0) / np.maximum(r, 0.05) / 3.0)
        v = rng.standard_normal((3, m)) * sig
        nk = int(kick_frac * m)
        if nk:
            k = rng.choice(m, nk, replace=False)
            kd = rng.standard_normal((3, nk))
            kd /= np.linalg.norm(kd, axis=0)
            v[:, k] += 3.0 * sig[k] * kd
        vs.append(v)
    return xs, vs


def lognormal_box(n_total, L, mesh, sigma=1.5, seed=0, device=None, slope=-2.0):
    """Poisson-like sample of a lognormal density field in a periodic box
    (the large-FoF configuration: 1024^3 particles, L = 1024, a 512^3 mesh,
    sigma_G = 1.5, P(k) ~ k^-2).

    A Gaussian field with power spectrum P(k) ~ k^slope on a mesh^3 grid,
    normalised to standard deviation sigma; weights exp(G - sigma^2/2) per
    mesh cell; cell counts drawn so that they sum to exactly n_total
    (Poisson counts of the expected numbers, then the difference spread over
    randomly chosen cells by weight); positions uniform inside their cell.

    With `device` (a torch device) the field, counts and positions are made
    there and a (3, n_total) float64 torch tensor is returned; otherwise a
    numpy array.  Both follow the same recipe but not the same random stream.
    """
    if device is None:
        rng = np.random.default_rng(seed)
        g = rng.standard_normal((mesh, mesh, mesh))
        gk = np.fft.rfftn(g)
        kx = np.fft.fftfreq(mesh)[:, None, None]
        ky = np.fft.fftfreq(mesh)[None, :, None]
        kz = np.fft.rfftfreq(mesh)[None, None, :]
        k2 = kx * kx + ky * ky + kz * kz
        k2[0, 0, 0] = np.inf
        gk *= np.power(k2, slope / 4.0)  # amplitude ~ sqrt(P) = k^(slope/2)
        g = np.fft.irfftn(gk, s=(mesh, mesh, mesh))
        g *= sigma / g.std()
        w = np.exp(g - 0.5 * sigma * sigma).ravel()
        lam = w * (n_total / w.sum())
        counts = rng.poisson(lam).astype(np.int64)
        diff = n_total - int(counts.sum())
        while diff != 0:
            idx = rng.choice(counts.size, size=abs(diff), p=w / w.sum())
            if diff > 0:
                np.add.at(counts, idx, 1)
            else:
                sub = np.bincount(idx, minlength=counts.size)
                counts = np.maximum(counts - sub, 0)
            diff = n_total - int(counts.sum())
        cells = np.repeat(np.arange(counts.size, dtype=np.int64), counts)
        cz, rem = np.divmod(cells, mesh * mesh)
        cy, cx = np.divmod(rem, mesh)
        h = L / mesh
        xp = np.empty((3, n_total))
        xp[0] = (cx + rng.random(n_total)) * h
        xp[1] = (cy + rng.random(n_total)) * h
        xp[2] = (cz + rng.random(n_total)) * h
        return np.mod(xp, L)
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    g = torch.randn((mesh, mesh, mesh), generator=gen, device=device, dtype=torch.float32)
    gk = torch.fft.rfftn(g)
    del g
    kx = torch.fft.fftfreq(mesh, device=device)[:, None, None]
    ky = torch.fft.fftfreq(mesh, device=device)[None, :, None]
    kz = torch.fft.rfftfreq(mesh, device=device)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = float("inf")
    gk *= torch.pow(k2, slope / 4.0)
    del k2
    g = torch.fft.irfftn(gk, s=(mesh, mesh, mesh))
    del gk
    g = g.double()
    g *= sigma / g.std()
    w = torch.exp(g - 0.5 * sigma * sigma).reshape(-1)
    del g
    lam = w * (n_total / w.sum())
    counts = torch.poisson(lam, generator=gen).long()
    diff = n_total - int(counts.sum().item())
    cdf = torch.cumsum(w, 0)
    while diff != 0:
        # cells drawn by weight (inverse of the cumulative weights)
        u = torch.rand(abs(diff), generator=gen, device=device, dtype=torch.float64) * cdf[-1]
        idx = torch.clamp(torch.searchsorted(cdf, u), max=counts.numel() - 1)
        sub = torch.bincount(idx, minlength=counts.numel())
        counts = counts + sub if diff > 0 else torch.clamp(counts - sub, min=0)
        diff = n_total - int(counts.sum().item())
    del lam, cdf, w
    # positions cell by cell, in slices of cells to bound the temporaries
    h = L / mesh
    xp = torch.empty((3, n_total), dtype=torch.float64, device=device)
    ends = torch.cumsum(counts, 0)
    starts = ends - counts
    ncell = counts.numel()
    step = 1 << 22
    for c0 in range(0, ncell, step):
        c1 = min(ncell, c0 + step)
        p0, p1 = int(starts[c0].item()), int(ends[c1 - 1].item())
        if p1 <= p0:
            continue
        cells = torch.repeat_interleave(torch.arange(c0, c1, device=device), counts[c0:c1])
        cz = torch.div(cells, mesh * mesh, rounding_mode="floor")
        rem = cells - cz * (mesh * mesh)
        cy = torch.div(rem, mesh, rounding_mode="floor")
        cx = rem - cy * mesh
        for d, c in enumerate((cx, cy, cz)):
            u = torch.rand(p1 - p0, generator=gen, device=device, dtype=torch.float64)
            xp[d, p0:p1] = torch.remainder((c.double() + u) * h, L)
    return xp
