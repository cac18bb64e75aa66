"""py_fof on NVIDIA B200: friends-of-friends halo finding with gravitational
unbinding, computed by hand-written sm_100a CUDA kernels.

Drop-in replacement of the reference package's public API
(py_fof/__init__.py): ``fof``, ``fof_with_info`` and the wrapper core
``_fof_core`` keep their signatures, argument validation, unit conversion,
error mapping and return values.  The compiled Fortran/f2py module is
replaced by the C-ABI library ``libpyfof_b200.so`` (include/pyfof_b200.h).
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from . import _native

__all__ = ["fof", "fof_with_info", "FofCall"]


@dataclass
class FofCall:
    """Arguments of one native call, after validation and unit conversion
    (the argument list of fof_fortran.fof_fortran, py_fof/__init__.py:331-335)."""
    xp: np.ndarray
    vp: np.ndarray | None
    mp: np.ndarray | None
    np_halo: np.ndarray
    nhalo: int
    L_Box: float
    link: float
    np_halo_min: int
    bound_check: int
    verbose: int
    softening: float
    a_val: float
    b_val: float
    s_15_val: float
    n_threads: int
    total_np: int
    ng_val: int
    ng_global_val: float
    ang_mom_scale: float
    # (x_div, v_mul, m_div, m_const): the conversion of xp/vp/mp to code
    # units that the device applies after the copy (pyfof_units_t); None
    # when the arrays above are in code units already
    units: tuple | None = None

    def on_host(self):
        """The same call with the unit conversion done here, in NumPy, as the
        reference does it (py_fof/__init__.py:302-321)."""
        if self.units is None:
            return self
        x_div, v_mul, m_div, m_const = self.units
        xp = self.xp if x_div == 1.0 else np.ascontiguousarray(self.xp / x_div, dtype=np.float64)
        vp = self.vp if (self.vp is None or v_mul == 1.0) else np.ascontiguousarray(self.vp * v_mul)
        if self.mp is not None:
            mp = self.mp if m_div == 1.0 else np.ascontiguousarray(self.mp / m_div, dtype=np.float64)
        else:
            mp = None if m_const == 1.0 else np.full(self.total_np, m_const, dtype=np.float64)
        return replace(self, xp=xp, vp=vp, mp=mp, units=None)

    def dense(self):
        """vp/mp in code units, materialised exactly as the reference passes them."""
        c = self.on_host()
        vp = c.vp if c.vp is not None else np.zeros((3, c.total_np), dtype=np.float64)
        mp = c.mp if c.mp is not None else np.ones(c.total_np, dtype=np.float64)
        return vp, mp


_MASS_ERROR = "All particle masses in mp_list must be positive and finite"


def _as_3n(xp_list_norm, staging=None):
    if len(xp_list_norm) == 1:
        x = xp_list_norm[0]
        if x.dtype == np.float64 and (x.flags.c_contiguous or x.flags.f_contiguous):
            return x
        return np.ascontiguousarray(x, dtype=np.float64)
    if staging is not None:
        out = staging.take((3, sum(x.shape[1] for x in xp_list_norm)))
        np.concatenate(xp_list_norm, axis=1, out=out)
        return out
    return np.ascontiguousarray(np.hstack(xp_list_norm), dtype=np.float64)


def _prepare(xp_list, vp_list=None, L_Box=512.0, linking_length=0.2, np_halo_min=10,
             bound_check=False, verbose=0, return_ang_mom=False, n_threads=None, mp_list=None,
             softening=None, z=0.0, box=300.0, h0=0.67, omega_m=0.3, omega_l=0.7, n_sim=None,
             units='cube', include_hubble_flow=False, ng=None, ng_global=None,
             check_masses=True, device_units=False, staging=None):
    """Validation and unit conversion of _fof_core (py_fof/__init__.py:168-329).

    Returns either a FofCall or, for total_np == 0, the final empty result.
    With check_masses=False the per-particle mass check (positive and
    finite) is left to the native library, which runs it on the device and
    reports it as ierr 5; _finish raises the same ValueError for it.
    `staging` (an _native.Staging): lists of regions are concatenated into
    its page-locked memory instead of new arrays; the arrays of the returned
    call are then valid until the staging's next use.
    With device_units=True the arrays stay in the caller's units and the
    call carries their conversion (FofCall.units), which the library applies
    on the device; a scalar mass then travels as that constant instead of
    an array of N copies.
    """
    if units not in ('cube', 'physical'):
        raise ValueError(f"units must be 'cube' or 'physical', got '{units}'")

    if n_threads is None or n_threads <= 0:
        n_threads_val = 0
    else:
        if n_threads > 256:
            raise ValueError("n_threads cannot exceed 256")
        n_threads_val = int(n_threads)

    if isinstance(xp_list, np.ndarray) and xp_list.ndim == 2:
        xp_list_norm = [xp_list]
    elif isinstance(xp_list, (list, tuple)):
        xp_list_norm = list(xp_list)
    else:
        raise ValueError("xp_list must be a 2D numpy array (3, N) or a list of 2D arrays")

    nhalo = len(xp_list_norm)
    for i, xp in enumerate(xp_list_norm):
        if not isinstance(xp, np.ndarray) or xp.ndim != 2 or xp.shape[0] != 3:
            raise ValueError(f"xp_list[{i}] must have shape (3, N), got {getattr(xp, 'shape', type(xp))}")

    np_halo = np.array([xp.shape[1] for xp in xp_list_norm], dtype=np.int32)
    total_np = int(np.sum(np_halo))

    if total_np == 0:
        return (np.zeros(0, dtype=bool), np.zeros(0, dtype=np.int32),
                np.zeros((3, nhalo), dtype=np.float64))

    if staging is not None:
        multi = len(xp_list_norm) > 1
        need = 24 * total_np if multi else 0
        if multi and isinstance(vp_list, (list, tuple)):
            need += 24 * total_np
        if isinstance(mp_list, (list, tuple)):
            need += 8 * total_np
        if not staging.reserve(need + 1024):
            staging = None
    xp_halo = _as_3n(xp_list_norm, staging)

    if bound_check and vp_list is None:
        raise ValueError("vp_list is required when bound_check=True")

    if vp_list is not None:
        if isinstance(vp_list, np.ndarray) and vp_list.ndim == 2:
            vp_list_norm = [vp_list]
        elif isinstance(vp_list, (list, tuple)):
            vp_list_norm = list(vp_list)
        else:
            raise ValueError("vp_list must be a 2D numpy array (3, N) or a list of 2D arrays")

        if len(vp_list_norm) != nhalo:
            raise ValueError(f"vp_list length ({len(vp_list_norm)}) must match xp_list length ({nhalo})")

        for i, vp in enumerate(vp_list_norm):
            if not isinstance(vp, np.ndarray) or vp.ndim != 2 or vp.shape != xp_list_norm[i].shape:
                raise ValueError(f"vp_list[{i}] shape {getattr(vp, 'shape', None)} must match xp_list[{i}] shape {xp_list_norm[i].shape}")

        vp_halo = _as_3n(vp_list_norm, staging)
    else:
        vp_halo = None  # the reference passes zeros (py_fof/__init__.py:233)

    mp_raw = None
    mp_scalar = None  # a scalar mass kept as such (device_units only)
    if mp_list is not None:
        if np.isscalar(mp_list) or (isinstance(mp_list, np.ndarray) and mp_list.ndim == 0):
            val = float(mp_list)
            if val <= 0 or not np.isfinite(val):
                raise ValueError("mp_list scalar must be positive and finite")
            if device_units:
                mp_scalar = val
            else:
                mp_raw = np.full(total_np, val, dtype=np.float64)
        elif isinstance(mp_list, np.ndarray):
            if mp_list.ndim == 1 and len(mp_list) == total_np:
                mp_raw = np.ascontiguousarray(mp_list, dtype=np.float64)
            elif nhalo > 1 and mp_list.ndim == 1 and len(mp_list) == nhalo:
                mp_raw = np.repeat(np.ascontiguousarray(mp_list, dtype=np.float64), np_halo)
            else:
                raise ValueError(f"mp_list 1D array length ({len(mp_list)}) does not match total particles ({total_np})")
        elif isinstance(mp_list, (list, tuple)):
            if len(mp_list) == nhalo and all(isinstance(m, np.ndarray) and m.ndim == 1 and len(m) == np_halo[i] for i, m in enumerate(mp_list)):
                if staging is not None:
                    mp_raw = staging.take((total_np,))
                    np.concatenate(mp_list, out=mp_raw)
                else:
                    mp_raw = np.concatenate(mp_list).astype(np.float64)
            elif len(mp_list) == nhalo and all(np.isscalar(m) for m in mp_list):
                scalars = np.array([float(m) for m in mp_list], dtype=np.float64)
                mp_raw = np.repeat(scalars, np_halo)
            elif len(mp_list) == total_np and all(np.isscalar(m) for m in mp_list):
                mp_raw = np.array(mp_list, dtype=np.float64)
            else:
                raise ValueError("mp_list structure does not match xp_list structure or particle counts")
        else:
            raise ValueError("Unsupported mp_list type")

        if check_masses and mp_raw is not None and (not np.all(np.isfinite(mp_raw)) or not np.all(mp_raw > 0)):
            raise ValueError(_MASS_ERROR)

    z_val = float(z)
    if 1.0 + z_val <= 0.0:
        raise ValueError(f"1 + z must be positive, got {1.0 + z_val}")
    a_val = 1.0 / (1.0 + z_val)

    if include_hubble_flow:
        t0 = 1.0 / (150.0 * float(h0) * np.sqrt(float(omega_m)))
        hubble = 100.0 * float(h0) * np.sqrt(float(omega_m) / (a_val ** 3) + float(omega_l))
        b_val = hubble * (a_val ** 2) * t0
    else:
        b_val = 0.0

    if units == 'cube':
        softening_grid = 0.1 if softening is None else float(softening)
        if bound_check and softening_grid <= 0:
            raise ValueError("softening must be positive")
        ng_eff_global = float(ng_global) if ng_global is not None else float(L_Box)
        s_15_val = 15.0 * float(h0) * ng_eff_global / float(box)
        xp_code = xp_halo
        L_Box_code = float(L_Box)
        link_code = float(linking_length)
        vp_code = vp_halo
        mp_code = mp_raw  # None means unit masses (py_fof/__init__.py:290-291)
        ang_mom_scale = 1.0
        conv = None if mp_scalar is None else (1.0, 1.0, 1.0, mp_scalar)
    else:
        if bound_check:
            if softening is None or float(softening) <= 0:
                raise ValueError("softening must be explicitly provided and > 0 when units='physical' and bound_check=True")
            if mp_raw is None and mp_scalar is None and n_sim is None:
                raise ValueError("Either mp_list or n_sim must be provided when units='physical' and bound_check=True")

        ng_eff = float(round(float(n_sim) ** (1.0 / 3.0))) if (n_sim is not None and float(n_sim) > 0) else (float(ng_global) if ng_global is not None else 512.0)
        box_mpc_h = float(L_Box)
        dx = box_mpc_h / ng_eff

        L_Box_code = ng_eff
        link_code = float(linking_length) / dx
        softening_grid = 0.1 if softening is None else (float(softening) / dx)
        s_15_val = 15.0 * float(h0) * ng_eff / box_mpc_h

        v_scale = (a_val * ng_eff) / (150.0 * np.sqrt(float(omega_m)) * box_mpc_h)

        rho_crit_0 = 2.77536627e11
        m_grid = float(omega_m) * rho_crit_0 * (box_mpc_h ** 3) / (ng_eff ** 3)

        if device_units:
            # the device divides/multiplies with the same IEEE operations
            xp_code, vp_code, mp_code = xp_halo, vp_halo, mp_raw
            if mp_raw is not None:
                conv = (dx, v_scale, m_grid, 1.0)
            elif mp_scalar is not None:
                conv = (dx, v_scale, 1.0, mp_scalar / m_grid)
            elif n_sim is not None:
                conv = (dx, v_scale, 1.0, (ng_eff ** 3) / float(n_sim))
            else:
                conv = (dx, v_scale, 1.0, 1.0)
                m_grid = 1.0
        else:
            conv = None
            xp_code = np.ascontiguousarray(xp_halo / dx, dtype=np.float64)
            vp_code = None if vp_halo is None else np.ascontiguousarray(vp_halo * v_scale, dtype=np.float64)
            if mp_raw is not None:
                mp_code = np.ascontiguousarray(mp_raw / m_grid, dtype=np.float64)
            elif n_sim is not None:
                mp_code = np.full(total_np, (ng_eff ** 3) / float(n_sim), dtype=np.float64)
            else:
                mp_code = None
                m_grid = 1.0

        ang_mom_scale = m_grid * dx / v_scale

    ng_val = int(ng) if ng is not None else 256
    ng_global_val = float(ng_global) if ng_global is not None else 512.0

    return FofCall(xp=xp_code, vp=vp_code, mp=mp_code, np_halo=np_halo, nhalo=nhalo,
                   L_Box=L_Box_code, link=link_code, np_halo_min=int(np_halo_min),
                   bound_check=int(bound_check), verbose=int(verbose), softening=softening_grid,
                   a_val=a_val, b_val=b_val, s_15_val=s_15_val, n_threads=n_threads_val,
                   total_np=total_np, ng_val=ng_val, ng_global_val=ng_global_val,
                   ang_mom_scale=ang_mom_scale, units=conv)


def _finish(call: FofCall, in_halo_out, halo_id_out, ang_mom_out, ierr):
    """ierr -> exception mapping and output conversion (py_fof/__init__.py:338-351)."""
    if ierr != 0:
        if ierr == 1:
            raise ValueError("Invalid input parameters or configuration in FOF/bound_test")
        elif ierr == 2:
            raise ValueError("Candidate halo span exceeds 15 Mpc limit (s_15)")
        elif ierr == 4:
            raise ValueError("Non-finite values (NaN/Inf) encountered during calculation")
        elif ierr == 5:
            raise ValueError(_MASS_ERROR)
        elif ierr == 10:
            raise ValueError("n_threads exceeds maximum supported slots (256)")
        else:
            detail = _native.last_error() if ierr == 20 else ""
            raise RuntimeError(f"FOF Fortran computation failed with error code ierr={ierr}"
                               + (f" ({detail})" if detail else ""))
    ang_mom_scaled = ang_mom_out * call.ang_mom_scale
    if in_halo_out.dtype != np.bool_:
        in_halo_out = in_halo_out.astype(bool)
    return in_halo_out, halo_id_out, ang_mom_scaled


def _native_call(call: FofCall, mask_only=False):
    return _native.run(call.xp, call.vp, call.mp, call.np_halo, call.nhalo, call.L_Box,
                       call.link, call.np_halo_min, call.bound_check, call.verbose,
                       call.softening, call.a_val, call.b_val, call.s_15_val, call.n_threads,
                       call.total_np, ng_val=call.ng_val, ng_global_val=call.ng_global_val,
                       units=call.units, mask_only=mask_only)


def _run_public(mask_only, **kw):
    """_prepare, the native call and _finish; with `mask_only` the library
    returns in_halo alone (halo_id is None), which is all fof() needs."""
    call = _prepare(check_masses=False, device_units=True, staging=_native.thread_staging(), **kw)
    if not isinstance(call, FofCall):
        return call
    in_halo, halo_id, ang_mom, ierr = _native_call(call, mask_only=mask_only)
    return _finish(call, in_halo, halo_id, ang_mom, ierr)


def _fof_core(xp_list, vp_list=None, L_Box=512.0, linking_length=0.2,
              np_halo_min=10, bound_check=False, verbose=0, return_ang_mom=False,
              n_threads=None, mp_list=None, softening=None, z=0.0,
              box=300.0, h0=0.67, omega_m=0.3, omega_l=0.7, n_sim=None,
              units='cube', include_hubble_flow=False,
              ng=None, ng_global=None):
    """Validation, unit conversion and the native call; returns
    (in_halo, halo_id, ang_mom) like the reference wrapper core."""
    return _run_public(False, xp_list=xp_list, vp_list=vp_list, L_Box=L_Box,
                       linking_length=linking_length, np_halo_min=np_halo_min,
                       bound_check=bound_check, verbose=verbose, return_ang_mom=return_ang_mom,
                       n_threads=n_threads, mp_list=mp_list, softening=softening, z=z, box=box,
                       h0=h0, omega_m=omega_m, omega_l=omega_l, n_sim=n_sim, units=units,
                       include_hubble_flow=include_hubble_flow, ng=ng, ng_global=ng_global)


def fof(xp_list, vp_list=None, L_Box=512.0, linking_length=0.2,
        np_halo_min=10, bound_check=False, verbose=0, return_ang_mom=False,
        n_threads=None, mp_list=None, softening=None, z=0.0,
        box=300.0, h0=0.67, omega_m=0.3, omega_l=0.7, n_sim=None,
        units='cube', include_hubble_flow=False,
        ng=None, ng_global=None):
    """Friends-of-friends halo finder (py_fof/__init__.py:354-447).

    Returns ``in_halo`` (bool, shape (total_np,)) and, with
    ``return_ang_mom=True``, the per-input-region angular momentum (3, nhalo).
    Parameters and units are those of the reference ``py_fof.fof``.
    """
    # the core of _fof_core with only in_halo crossing back from the device
    in_halo, _, ang_mom = _run_public(
        True, xp_list=xp_list, vp_list=vp_list, L_Box=L_Box, linking_length=linking_length,
        np_halo_min=np_halo_min, bound_check=bound_check, verbose=verbose,
        return_ang_mom=return_ang_mom, n_threads=n_threads, mp_list=mp_list,
        softening=softening, z=z, box=box, h0=h0, omega_m=omega_m, omega_l=omega_l,
        n_sim=n_sim, units=units, include_hubble_flow=include_hubble_flow,
        ng=ng, ng_global=ng_global
    )
    if return_ang_mom:
        return in_halo, ang_mom
    return in_halo


def catalogue_from_ids(in_halo, halo_id, ang_mom=None, return_ang_mom=False):
    """Halo catalogue of fof_with_info (py_fof/__init__.py:481-518)."""
    total_np = len(halo_id)
    max_id = int(np.max(halo_id)) if total_np > 0 else 0

    if max_id == 0:
        nhalo_found = 0
        np_per_halo = np.array([], dtype=int)
        halo_indices = []
    else:
        valid_mask = (halo_id > 0)
        valid_indices = np.where(valid_mask)[0]
        valid_hids = halo_id[valid_indices]
        counts = np.bincount(valid_hids, minlength=max_id + 1)[1:max_id + 1]
        order = np.argsort(valid_hids, kind='stable')
        sorted_indices = valid_indices[order]
        split_points = np.cumsum(counts)[:-1]
        raw_splits = np.split(sorted_indices, split_points) if len(split_points) > 0 else [sorted_indices]
        halo_indices = [idx for idx, c in zip(raw_splits, counts) if c > 0]
        np_per_halo = counts[counts > 0]
        nhalo_found = len(halo_indices)

    res = {
        'in_halo': in_halo,
        'nhalo_found': nhalo_found,
        'np_per_halo': np_per_halo,
        'halo_indices': halo_indices,
        'bound_status': np.zeros(nhalo_found, dtype=np.int32)
    }
    if return_ang_mom:
        res['ang_mom'] = ang_mom
    return res


def fof_with_info(xp_list, vp_list=None, L_Box=512.0, linking_length=0.2,
                  np_halo_min=10, bound_check=False, verbose=0, return_ang_mom=False,
                  n_threads=None, mp_list=None, softening=None, z=0.0,
                  box=300.0, h0=0.67, omega_m=0.3, omega_l=0.7, n_sim=None,
                  units='cube', include_hubble_flow=False,
                  ng=None, ng_global=None):
    """FoF with a halo catalogue (py_fof/__init__.py:450-518).

    Returns a dict with 'in_halo', 'nhalo_found', 'np_per_halo',
    'halo_indices' (ascending particle indices per halo, ordered by halo id),
    'bound_status' (zeros) and, if requested, 'ang_mom'.
    """
    call = _prepare(xp_list, vp_list=vp_list, L_Box=L_Box, linking_length=linking_length,
                    np_halo_min=np_halo_min, bound_check=bound_check, verbose=verbose,
                    return_ang_mom=return_ang_mom, n_threads=n_threads, mp_list=mp_list,
                    softening=softening, z=z, box=box, h0=h0, omega_m=omega_m,
                    omega_l=omega_l, n_sim=n_sim, units=units,
                    include_hubble_flow=include_hubble_flow, ng=ng, ng_global=ng_global,
                    check_masses=False, device_units=True, staging=_native.thread_staging())
    if not isinstance(call, FofCall):
        return catalogue_from_ids(*call, return_ang_mom=return_ang_mom)
    return _catalogue_call(call, return_ang_mom)


def _catalogue_call(call: FofCall, return_ang_mom, slot=None):
    """One native call with the catalogue sorted on the device; the result
    dict of fof_with_info (py_fof/__init__.py:481-518)."""
    ih, hid, am, ierr, members, offsets = _native.run_catalogue(
        call.xp, call.vp, call.mp, call.np_halo, call.nhalo, call.L_Box, call.link, call.np_halo_min,
        call.bound_check, call.verbose, call.softening, call.a_val, call.b_val, call.s_15_val,
        call.n_threads, call.total_np, ng_val=call.ng_val, ng_global_val=call.ng_global_val, slot=slot,
        units=call.units)
    in_halo, _, ang_mom = _finish(call, ih, hid, am, ierr)
    counts = np.diff(offsets)
    if counts.size == 0:
        halo_indices, np_per_halo = [], np.array([], dtype=int)
    else:
        halo_indices = np.split(members.astype(np.int64), offsets[1:-1])
        np_per_halo = counts
        if not np.all(counts > 0):  # ids without members are not listed
            halo_indices = [h for h, c in zip(halo_indices, counts) if c > 0]
            np_per_halo = counts[counts > 0]
    nfound = len(halo_indices)
    res = {
        'in_halo': in_halo,
        'nhalo_found': nfound,
        'np_per_halo': np_per_halo,
        'halo_indices': halo_indices,
        'bound_status': np.zeros(nfound, dtype=np.int32)
    }
    if return_ang_mom:
        res['ang_mom'] = ang_mom
    return res
