"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``liboracle.so``, built from this directory's C sources by
``make -C oracle``) restates the reference's friends-of-friends and
unbinding algorithms on the CPU.  Only the test-suite, the smoke check and
the CPU-baseline leg of ``bench.py`` may load it; the product package
``py_fof_b200`` never imports this module.

``fof_fortran`` mirrors the f2py signature of the reference extension
(fof_fortran.f90:10-13): it takes (3,N) float64 arrays and returns
``(in_halo, halo_id, ang_mom, ierr)``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build() -> str:
    """Compile liboracle.so in place (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_fof_fortran.restype = ctypes.c_int32
        L.oracle_fof_fortran.argtypes = [
            _dp, _dp, _dp, _i32p, ctypes.c_int32, ctypes.c_int64,
            ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_int32, ctypes.c_int64, ctypes.c_double, _i32p, _i32p, _dp]
        L.oracle_fof_fortran_diag.restype = ctypes.c_int32
        L.oracle_fof_fortran_diag.argtypes = L.oracle_fof_fortran.argtypes + [_fp, _fp]
        L.oracle_last_threads.restype = ctypes.c_int32
        L.oracle_bound_batch.restype = ctypes.c_int32
        L.oracle_bound_batch.argtypes = [
            _fp, _fp, _i64p, _i32p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
            ctypes.c_int64, ctypes.c_double, _i32p, _i32p, _i32p, _fp, _i32p]
        L.oracle_bound_first_potential.restype = ctypes.c_int32
        L.oracle_bound_first_potential.argtypes = [
            _fp, _fp, _i64p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_int64, _fp]
        L.oracle_direct_potential_f64.restype = None
        L.oracle_direct_potential_f64.argtypes = [_fp, _fp, ctypes.c_int32, ctypes.c_double,
                                                  ctypes.c_double, _dp]
        L.oracle_green_and_self.restype = ctypes.c_int32
        L.oracle_green_and_self.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_int32, _fp, _fp]
        L.oracle_modulo.restype = ctypes.c_double
        L.oracle_modulo.argtypes = [ctypes.c_double, ctypes.c_double]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def fof_fortran(xp_halo, vp_halo, mp_halo, np_halo, nhalo, L_Box, linking_length,
                np_halo_min, bound_check, verbose, softening, a_val, b_val, s_15_val,
                n_threads, total_np, ng_val=256, ng_global_val=512.0, diag=False):
    """Oracle counterpart of the f2py entry ``fof_fortran.fof_fortran``.

    With ``diag=True`` it also returns the unbinding diagnostics
    ``energy`` (each candidate member's specific energy at its last
    evaluation in the removal loop) and ``phi_scale`` (max |phi| of its
    candidate's first-pass potential), float32 per particle, NaN outside
    candidates."""
    xp = np.asfortranarray(xp_halo, dtype=np.float64)
    vp = np.asfortranarray(vp_halo, dtype=np.float64)
    mp = np.ascontiguousarray(mp_halo, dtype=np.float64)
    nph = np.ascontiguousarray(np_halo, dtype=np.int32)
    n = int(total_np)
    in_halo = np.zeros(n, dtype=np.int32)
    halo_id = np.zeros(n, dtype=np.int32)
    ang_mom = np.zeros((3, max(int(nhalo), 0)), dtype=np.float64, order="F")
    args = [_p(xp, _dp), _p(vp, _dp), _p(mp, _dp), _p(nph, _i32p), int(nhalo), n,
            float(L_Box), float(linking_length), int(np_halo_min), int(bound_check), int(verbose),
            float(softening), float(a_val), float(b_val), float(s_15_val), int(n_threads),
            int(ng_val), float(ng_global_val), _p(in_halo, _i32p), _p(halo_id, _i32p),
            _p(ang_mom, _dp)]
    if not diag:
        ierr = lib().oracle_fof_fortran(*args)
        return in_halo, halo_id, ang_mom, int(ierr)
    energy = np.zeros(n, np.float32)
    phi_scale = np.zeros(n, np.float32)
    ierr = lib().oracle_fof_fortran_diag(*args, _p(energy, _fp), _p(phi_scale, _fp))
    return in_halo, halo_id, ang_mom, int(ierr), energy, phi_scale


def last_threads() -> int:
    return int(lib().oracle_last_threads())


def bound_batch(xv, mp, pid, cand_np, softening=0.1, a_val=1.0, b_val=0.0, s15=17.152,
                np_halo_min=10, verbose=0, n_threads=0, ng_val=256, ng_global_val=512.0,
                want_phi=False):
    """Unbinding of pre-packed candidates; returns (ierr, np_bound, status,
    final_members, phi or None, method)."""
    xv = np.ascontiguousarray(xv, dtype=np.float32)  # (N,6) rows = xv(:,i)
    mp = np.ascontiguousarray(mp, dtype=np.float32)
    pid = np.ascontiguousarray(pid, dtype=np.int64)
    cnp = np.ascontiguousarray(cand_np, dtype=np.int32)
    nc = len(cnp)
    nb = np.zeros(nc, np.int32)
    st = np.zeros(nc, np.int32)
    fm = np.zeros(len(pid), np.int32)
    meth = np.zeros(nc, np.int32)
    phi = np.zeros(len(pid), np.float32) if want_phi else None
    ierr = lib().oracle_bound_batch(
        _p(xv, _fp), _p(mp, _fp), _p(pid, _i64p), _p(cnp, _i32p), nc, float(softening),
        float(a_val), float(b_val), float(s15), int(np_halo_min), int(verbose), int(n_threads),
        int(ng_val), float(ng_global_val), _p(nb, _i32p), _p(st, _i32p), _p(fm, _i32p),
        _p(phi, _fp) if phi is not None else None, _p(meth, _i32p))
    return int(ierr), nb, st, fm, phi, meth


def first_potential(xv, mp, pid, softening=0.1, a_val=1.0, s15=17.152, ng_val=256):
    xv = np.ascontiguousarray(xv, dtype=np.float32)
    mp = np.ascontiguousarray(mp, dtype=np.float32)
    pid = np.ascontiguousarray(pid, dtype=np.int64)
    phi = np.zeros(len(pid), np.float32)
    g = lib().oracle_bound_first_potential(_p(xv, _fp), _p(mp, _fp), _p(pid, _i64p), len(pid),
                                           float(softening), float(a_val), float(s15),
                                           int(ng_val), _p(phi, _fp))
    return int(g), phi


def direct_potential_f64(q, w, softening=0.1, a_val=1.0):
    q = np.ascontiguousarray(q, dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    phi = np.zeros(len(w), np.float64)
    lib().oracle_direct_potential_f64(_p(q, _fp), _p(w, _fp), len(w), float(softening),
                                      float(a_val), _p(phi, _dp))
    return phi


def green_and_self(n, apm_soft=3.5, apm_range=0.0, truncated=True):
    g = np.zeros((n, n, n // 2 + 1), np.float32)
    s = np.zeros((5, 5, 5), np.float32)
    e = lib().oracle_green_and_self(int(n), float(apm_soft), float(apm_range), int(truncated),
                                    _p(g, _fp), _p(s, _fp))
    if e:
        raise RuntimeError("oracle green failed")
    return g, s


def modulo(a, p):
    return lib().oracle_modulo(float(a), float(p))
