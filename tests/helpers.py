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
