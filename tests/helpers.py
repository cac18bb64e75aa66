"""Shared test helpers: the oracle-backed wrapper core, golden fixtures and
partition canonicalisation."""
from __future__ import annotations

import os

import numpy as np

from oracle import oracle as O
import py_fof_b200 as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LINK = 2.0
L_BOX = 512.0
NP_MIN = 10


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def oracle_core(xp_list, **kw):
    """_fof_core with the CPU oracle in place of the native call: the same
    validation/unit code (py_fof_b200._prepare/_finish), the reference
    algorithm restated in C."""
    call = P._prepare(xp_list, **kw)
    if not isinstance(call, P.FofCall):
        return call
    vp, mp = call.dense()
    xp = np.asfortranarray(call.xp)
    in_halo, halo_id, ang_mom, ierr = O.fof_fortran(
        xp, np.asfortranarray(vp), mp, call.np_halo, call.nhalo, call.L_Box, call.link,
        call.np_halo_min, call.bound_check, call.verbose, call.softening, call.a_val,
        call.b_val, call.s_15_val, call.n_threads, call.total_np, call.ng_val,
        call.ng_global_val)
    return P._finish(call, in_halo, halo_id, ang_mom, ierr)


def oracle_core_diag(xp_list, **kw):
    """oracle_core plus the unbinding diagnostics: returns ((in_halo,
    halo_id, ang_mom), energy, phi_scale) with energy = each candidate
    member's specific energy at its last evaluation in the oracle's removal
    loop and phi_scale = max |phi| of its candidate (NaN elsewhere)."""
    call = P._prepare(xp_list, **kw)
    vp, mp = call.dense()
    xp = np.asfortranarray(call.xp)
    in_halo, halo_id, ang_mom, ierr, energy, scale = O.fof_fortran(
        xp, np.asfortranarray(vp), mp, call.np_halo, call.nhalo, call.L_Box, call.link,
        call.np_halo_min, call.bound_check, call.verbose, call.softening, call.a_val,
        call.b_val, call.s_15_val, call.n_threads, call.total_np, call.ng_val,
        call.ng_global_val, diag=True)
    return P._finish(call, in_halo, halo_id, ang_mom, ierr), energy, scale


# Unbinding parity band.  A particle's specific energy E decides its
# membership (bound iff E < 0, bound_fortran.f90:2773-2786).  The FP32
# product path and the particle-mesh path (the oracle's FFT is not FFTW's)
# compute potentials that differ from the oracle's by up to ~1e-5 of the
# halo's largest |phi|, so only particles with |E| within a band around zero
# may be classified differently.  The band is ENERGY_BAND * max|phi| of the
# particle's candidate (first pass), with E the oracle's energy at the
# particle's last evaluation.
ENERGY_BAND = 1e-3


def check_unbinding_band(g, o, energy, scale, tau=ENERGY_BAND):
    """g, o: (in_halo, halo_id, ...) of the GPU and the oracle.  Asserts the
    same number of valid halos, the same halo ids wherever both keep a
    particle, and |E| <= tau * max|phi| for every particle classified
    differently.  Returns (number of flips, largest |E| / max|phi| among
    them)."""
    gi = np.asarray(g[0], bool)
    oi = np.asarray(o[0], bool)
    assert int(g[1].max()) == int(o[1].max()), (int(g[1].max()), int(o[1].max()))
    both = gi & oi
    assert np.array_equal(g[1][both], o[1][both])
    flip = np.nonzero(gi != oi)[0]
    worst = 0.0
    if flip.size:
        e = energy[flip].astype(np.float64)
        sc = scale[flip].astype(np.float64)
        assert np.all(np.isfinite(e)) and np.all(sc > 0)
        rel = np.abs(e) / sc
        worst = float(rel.max())
        assert worst <= tau, (flip.size, worst, tau)
    return int(flip.size), worst


def host_ang_mom(xp_list, vp_list, mp_list, L, halo_id):
    """Angular momentum per input region from a membership, in FP64 on the
    host, the reference's formula (fof_fortran.f90:224-248): members unwrapped
    about a member (MODULO), mass-weighted centre and bulk velocity, sum of
    m (dx - qc) x (v - vc).  Returns (ang_mom (3, nregion), term scale per
    region = sum of |m (dx - qc)| |v - vc|)."""
    if isinstance(xp_list, np.ndarray):
        xp_list, vp_list = [xp_list], [vp_list]
        mp_list = None if mp_list is None else [mp_list]
    out = np.zeros((3, len(xp_list)))
    scale = np.zeros(len(xp_list))
    off = 0
    half = 0.5 * L
    for r, x in enumerate(xp_list):
        n = x.shape[1]
        hid = halo_id[off:off + n]
        v = vp_list[r]
        m = np.ones(n) if mp_list is None or mp_list[r] is None else np.asarray(mp_list[r], float)
        if np.ndim(m) == 0:
            m = np.full(n, float(m))
        for h in np.unique(hid[hid > 0]):
            idx = np.nonzero(hid == h)[0]
            xa = x[:, idx[:1]]
            dx = O_modulo(x[:, idx] - xa + half, L) - half
            w = m[idx]
            qc = (dx * w).sum(axis=1, keepdims=True) / w.sum()
            vc = (v[:, idx] * w).sum(axis=1, keepdims=True) / w.sum()
            a = (dx - qc) * w
            b = v[:, idx] - vc
            out[:, r] += np.cross(a.T, b.T).sum(axis=0)
            scale[r] += float((np.linalg.norm(a, axis=0) * np.linalg.norm(b, axis=0)).sum())
        off += n
    return out, scale


def O_modulo(a, p):
    r = np.fmod(a, p)
    return np.where((r != 0.0) & ((r < 0.0) != (p < 0.0)), r + p, r)


def check_ang_mom_consistent(res, xp_list, vp_list, mp_list, L, rtol=1e-9):
    """ang_mom of a result equals the FP64 host sum over that result's own
    members within rtol of the summed terms' magnitude (only the summation
    order differs)."""
    ref, scale = host_ang_mom(xp_list, vp_list, mp_list, L, np.asarray(res[1]))
    am = np.asarray(res[2])
    assert np.all(np.abs(am - ref) <= rtol * (np.abs(ref) + scale[None, :] + 1e-300)), \
        float(np.max(np.abs(am - ref) / (np.abs(ref) + scale[None, :] + 1e-300)))


def oracle_fof(xp_list, return_ang_mom=False, **kw):
    in_halo, _, am = oracle_core(xp_list, return_ang_mom=return_ang_mom, **kw)
    return (in_halo, am) if return_ang_mom else in_halo


def oracle_fof_with_info(xp_list, return_ang_mom=False, **kw):
    in_halo, halo_id, am = oracle_core(xp_list, return_ang_mom=return_ang_mom, **kw)
    return P.catalogue_from_ids(in_halo, halo_id, am, return_ang_mom)


def canonical(halo_id):
    """Relabel groups by their minimum particle index (0 = no group)."""
    halo_id = np.asarray(halo_id)
    out = np.zeros_like(halo_id)
    ids = np.unique(halo_id[halo_id > 0])
    for h in ids:
        idx = np.nonzero(halo_id == h)[0]
        out[idx] = idx[0] + 1
    return out


def angmom_close(a, b, scale, rtol=1e-9):
    """Angular momenta agree up to summation-order rounding: |a-b| <=
    rtol * (|b| + scale), where scale bounds the summed terms' magnitude."""
    a = np.asarray(a)
    b = np.asarray(b)
    return np.all(np.abs(a - b) <= rtol * (np.abs(b) + scale))
