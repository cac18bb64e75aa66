"""ctypes binding of libpyfof_b200.so (declarations in include/pyfof_b200.h).

The shared library is built in place by ``python -m py_fof_b200.build``.
There is no fallback: if the library is missing or cannot be loaded, every
call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpyfof_b200.so")
ABI_VERSION = 2
LAYOUT_AOS = 0
LAYOUT_SOA = 1

_lib = None
_lock = threading.Lock()

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)

_RUN_ARGS = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, _i32p,
             ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
             ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
             ctypes.c_double, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p,
             ctypes.c_void_p, _dp]

class Units(ctypes.Structure):
    """pyfof_units_t: conversion of the inputs to code units on the device
    (positions / x_div, velocities * v_mul, masses / m_div, or m_const for
    every particle when there is no mass array)."""
    _fields_ = [("x_div", ctypes.c_double), ("v_mul", ctypes.c_double),
                ("m_div", ctypes.c_double), ("m_const", ctypes.c_double)]


def _units_ptr(units):
    return None if units is None else ctypes.byref(Units(*[float(v) for v in units]))


# every symbol include/pyfof_b200.h declares
EXPORTED = ("pyfof_version", "pyfof_init", "pyfof_shutdown", "pyfof_last_error",
            "pyfof_set_option", "pyfof_get_option", "pyfof_set_tile", "pyfof_get_tile", "pyfof_set_stream", "pyfof_get_stat", "pyfof_last_link_ms", "pyfof_last_stage_ms",
            "pyfof_halo_potential", "pyfof_halo_potential_direct_static", "pyfof_run",
            "pyfof_run_device", "pyfof_slot_create", "pyfof_slot_destroy", "pyfof_slot_run",
            "pyfof_slot_stat", "pyfof_run_catalogue", "pyfof_run_units", "pyfof_run_mask",
            "pyfof_host_alloc", "pyfof_host_free")


class NativeLibraryError(RuntimeError):
    pass


def load():
    """Load the library (once) and declare the C-ABI signatures."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryError(
                f"{LIB_PATH} is missing; build it with `python -m py_fof_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.pyfof_version.restype = ctypes.c_int32
        L.pyfof_init.restype = ctypes.c_int32
        L.pyfof_init.argtypes = [ctypes.c_int32]
        L.pyfof_shutdown.restype = ctypes.c_int32
        L.pyfof_last_error.restype = ctypes.c_int32
        L.pyfof_last_error.argtypes = [ctypes.c_char_p, ctypes.c_int64]
        L.pyfof_set_option.restype = ctypes.c_int32
        L.pyfof_set_option.argtypes = [ctypes.c_char_p, ctypes.c_int64]
        L.pyfof_get_option.restype = ctypes.c_int32
        L.pyfof_get_option.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.pyfof_set_tile.restype = ctypes.c_int32
        L.pyfof_set_tile.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64]
        L.pyfof_get_tile.restype = ctypes.c_int32
        L.pyfof_get_tile.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L.pyfof_set_stream.restype = ctypes.c_int32
        L.pyfof_set_stream.argtypes = [ctypes.c_void_p]
        L.pyfof_get_stat.restype = ctypes.c_int32
        L.pyfof_get_stat.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.pyfof_last_link_ms.restype = ctypes.c_int32
        L.pyfof_last_link_ms.argtypes = [ctypes.POINTER(ctypes.c_float)]
        L.pyfof_last_stage_ms.restype = ctypes.c_int32
        L.pyfof_last_stage_ms.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_float)]
        L.pyfof_halo_potential.restype = ctypes.c_int32
        L.pyfof_halo_potential.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_int32)]
        L.pyfof_halo_potential_direct_static.restype = ctypes.c_int32
        L.pyfof_halo_potential_direct_static.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
            ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
        L.pyfof_run.restype = ctypes.c_int32
        L.pyfof_run.argtypes = _RUN_ARGS
        L.pyfof_run_device.restype = ctypes.c_int32
        L.pyfof_run_device.argtypes = _RUN_ARGS
        L.pyfof_slot_create.restype = ctypes.c_int32
        L.pyfof_slot_create.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]
        L.pyfof_slot_destroy.restype = ctypes.c_int32
        L.pyfof_slot_destroy.argtypes = [ctypes.c_void_p]
        L.pyfof_slot_run.restype = ctypes.c_int32
        L.pyfof_slot_run.argtypes = [ctypes.c_void_p] + list(_RUN_ARGS)
        L.pyfof_run_catalogue.restype = ctypes.c_int32
        L.pyfof_run_units.restype = ctypes.c_int32
        L.pyfof_run_units.argtypes = [ctypes.c_void_p, ctypes.POINTER(Units)] + list(_RUN_ARGS)
        L.pyfof_run_mask.restype = ctypes.c_int32
        L.pyfof_run_mask.argtypes = ([ctypes.c_void_p, ctypes.POINTER(Units)] + list(_RUN_ARGS[:19]) +
                                     [ctypes.c_void_p, _dp])
        L.pyfof_run_catalogue.argtypes = ([ctypes.c_void_p, ctypes.POINTER(Units)] + list(_RUN_ARGS[:19]) +
                                          [_RUN_ARGS[20], _RUN_ARGS[21], ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32)])
        L.pyfof_host_alloc.restype = ctypes.c_int32
        L.pyfof_host_alloc.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]
        L.pyfof_host_free.restype = ctypes.c_int32
        L.pyfof_host_free.argtypes = [ctypes.c_void_p]
        L.pyfof_slot_stat.restype = ctypes.c_int32
        L.pyfof_slot_stat.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        v = L.pyfof_version()
        if v != ABI_VERSION:
            raise NativeLibraryError(f"ABI version mismatch: library {v}, binding {ABI_VERSION}")
        _lib = L
    apply_tile_table()
    return L


def last_error() -> str:
    L = load()
    buf = ctypes.create_string_buffer(2048)
    L.pyfof_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def set_option(key: str, value: int) -> None:
    if load().pyfof_set_option(key.encode(), int(value)) != 0:
        raise ValueError(last_error())


def get_option(key: str) -> int:
    v = ctypes.c_int64(0)
    if load().pyfof_get_option(key.encode(), ctypes.byref(v)) != 0:
        raise ValueError(last_error())
    return int(v.value)


# the tile table the autotuner writes (py_fof_b200.autotune); the
# environment variable PYFOF_TILE_TABLE names another file ("" = none)
TILE_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tiles.json")
TILE_KEYS = ("direct_threads", "pm_batch", "conv_waves")
_tile_table_used = None


def set_tile(key: str, index: int, value: int) -> None:
    if load().pyfof_set_tile(key.encode(), int(index), int(value)) != 0:
        raise ValueError(last_error())


def get_tile(key: str, index: int) -> int:
    v = ctypes.c_int64(0)
    if load().pyfof_get_tile(key.encode(), int(index), ctypes.byref(v)) != 0:
        raise ValueError(last_error())
    return int(v.value)


def read_tile_table(path):
    """Entries [(key, index, value)] of a tile table file (JSON: {key:
    {index: value}} for the keys of TILE_KEYS; other top-level keys are
    notes).  Raises ValueError on a malformed table."""
    import json
    with open(path) as f:
        d = json.load(f)
    if not isinstance(d, dict):
        raise ValueError(f"{path}: not a JSON object")
    out = []
    for key in TILE_KEYS:
        ent = d.get(key, {})
        if not isinstance(ent, dict):
            raise ValueError(f"{path}: {key} must map indices to values")
        for idx, val in ent.items():
            out.append((key, int(idx), int(val)))
    return out


def apply_tile_table(path=None):
    """Set the library's tile table from `path` (default: PYFOF_TILE_TABLE or
    the package's tiles.json when present).  Returns the path used or None."""
    global _tile_table_used
    if path is None:
        path = os.environ.get("PYFOF_TILE_TABLE", TILE_TABLE)
    if not path or not os.path.exists(path):
        return None
    for key, idx, val in read_tile_table(path):
        if _lib.pyfof_set_tile(key.encode(), idx, val) != 0:
            raise ValueError(f"{path}: {last_error()}")
    _tile_table_used = path
    return path


def tile_table_used():
    load()
    return _tile_table_used


class tiles:
    """Context manager: set tile-table entries, restore them after.

        with _native.tiles(("direct_threads", 0, 32)):
            ...
    """

    def __init__(self, *entries):
        self.entries = entries
        self.old = []

    def __enter__(self):
        for key, idx, val in self.entries:
            self.old.append((key, idx, get_tile(key, idx)))
            set_tile(key, idx, val)
        return self

    def __exit__(self, *exc):
        for key, idx, val in reversed(self.old):
            set_tile(key, idx, val)
        return False


class options:
    """Context manager: set library options, restore their values after.

        with _native.options(unbind_fp64=0):
            ...
    """

    def __init__(self, **opts):
        self.opts = opts
        self.old = {}

    def __enter__(self):
        for k, v in self.opts.items():
            self.old[k] = get_option(k)
            set_option(k, v)
        return self

    def __exit__(self, *exc):
        for k, v in self.old.items():
            set_option(k, v)
        return False


def set_stream(stream_handle: int) -> None:
    """Issue library work on the given cudaStream_t (0 = library stream)."""
    if load().pyfof_set_stream(ctypes.c_void_p(stream_handle) if stream_handle else None) != 0:
        raise RuntimeError(last_error())


def get_stat(key: str) -> int:
    v = ctypes.c_int64(0)
    if load().pyfof_get_stat(key.encode(), ctypes.byref(v)) != 0:
        raise ValueError(last_error())
    return int(v.value)


def last_link_ms() -> float:
    v = ctypes.c_float(0.0)
    load().pyfof_last_link_ms(ctypes.byref(v))
    return float(v.value)


def last_stage_ms(stage: str) -> float:
    """Device time of one stage of the last call ("link", "fof", "unbind",
    "call", "pm_fft"; after a host-memory call also "h2d_positions",
    "h2d_inputs", "d2h", "host_call"); needs set_option("timing", 1)."""
    v = ctypes.c_float(0.0)
    if load().pyfof_last_stage_ms(stage.encode(), ctypes.byref(v)) != 0:
        raise ValueError(last_error())
    return float(v.value)


class Staging:
    """Page-locked host memory that list inputs are concatenated into
    (pyfof_host_alloc), one per thread (thread_staging).  Views handed out
    by take() are valid until the next reserve() of the same object, which
    the public calls make at their start: the previous call of the thread
    has returned by then."""

    def __init__(self):
        self.ptr = None
        self.cap = 0
        self.used = 0

    def reserve(self, nbytes):
        """Room for `nbytes`; False when no page-locked memory could be had
        (the caller then concatenates into ordinary arrays)."""
        self.used = 0
        if nbytes <= self.cap:
            return True
        L = load()
        self.release()
        cap = max(int(nbytes), 1 << 20)
        p = ctypes.c_void_p()
        if L.pyfof_host_alloc(cap, ctypes.byref(p)) != 0:
            return False
        self.ptr, self.cap = p.value, cap
        return True

    def take(self, shape):
        """A float64 array of `shape` in the reserved memory (C order)."""
        n = int(np.prod(shape))
        off = (self.used + 255) // 256 * 256
        if off + 8 * n > self.cap:
            raise MemoryError("staging reservation exceeded")
        self.used = off + 8 * n
        buf = (ctypes.c_double * n).from_address(self.ptr + off)
        return np.frombuffer(buf, dtype=np.float64, count=n).reshape(shape)

    def release(self):
        if self.ptr is not None and _lib is not None:
            _lib.pyfof_host_free(ctypes.c_void_p(self.ptr))
        self.ptr, self.cap, self.used = None, 0, 0

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


_tls = threading.local()


def thread_staging():
    """The calling thread's Staging."""
    st = getattr(_tls, "staging", None)
    if st is None:
        st = _tls.staging = Staging()
    return st


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def run(xp, vp, mp, np_halo, nhalo, L_Box, link, np_halo_min, bound_check, verbose, softening,
        a_val, b_val, s_15_val, n_threads, total_np, ng_val=256, ng_global_val=512.0, slot=None,
        units=None, mask_only=False):
    """Host-memory call with the f2py argument order of fof_fortran.fof_fortran.

    xp, vp: (3,N) float64 arrays, C- or Fortran-contiguous (vp may be None);
    mp: (N,) float64 or None.  `slot`: a handle of slot_create, else the
    default context.  `units`: (x_div, v_mul, m_div, m_const), the inputs'
    conversion to code units done on the device, or None.  Returns
    (in_halo, halo_id, ang_mom, ierr); with `mask_only` the library returns
    in_halo alone, as bytes written into a numpy bool array, and halo_id is
    None (pyfof_run_mask).
    """
    L = load()
    n = int(total_np)
    if xp.flags.c_contiguous:
        layout = LAYOUT_SOA
    elif xp.flags.f_contiguous:
        layout = LAYOUT_AOS
    else:
        xp = np.ascontiguousarray(xp)
        layout = LAYOUT_SOA
    if vp is not None:
        vp = np.asarray(vp, dtype=np.float64)
        vp = np.ascontiguousarray(vp) if layout == LAYOUT_SOA else np.asfortranarray(vp)
    if mp is not None:
        mp = np.ascontiguousarray(mp, dtype=np.float64)
    nph = np.ascontiguousarray(np_halo, dtype=np.int32)
    # written in full by the library (zeros on every failure path); in_halo
    # is halo_id > 0, so only halo_id crosses back to the host
    in_halo = None
    ang_mom = np.zeros((3, max(int(nhalo), 0)), dtype=np.float64, order="F")
    args = (_ptr(xp), _ptr(vp), _ptr(mp), layout, nph.ctypes.data_as(_i32p),
            int(nhalo), n, float(L_Box), float(link), int(np_halo_min),
            int(bound_check), int(verbose), float(softening), float(a_val),
            float(b_val), float(s_15_val), int(n_threads), int(ng_val),
            float(ng_global_val))
    if mask_only:
        in_halo = np.empty(n, dtype=np.bool_)
        ierr = L.pyfof_run_mask(ctypes.c_void_p(slot) if slot else None,
                                None if units is None else _units_ptr(units), *args,
                                _ptr(in_halo), ang_mom.ctypes.data_as(_dp))
        return in_halo, None, ang_mom, int(ierr)
    halo_id = np.empty(n, dtype=np.int32)
    args = args + (None, _ptr(halo_id), ang_mom.ctypes.data_as(_dp))
    if units is not None:
        ierr = L.pyfof_run_units(ctypes.c_void_p(slot) if slot else None, _units_ptr(units), *args)
    elif slot is None:
        ierr = L.pyfof_run(*args)
    else:
        ierr = L.pyfof_slot_run(ctypes.c_void_p(slot), *args)
    in_halo = halo_id > 0
    return in_halo, halo_id, ang_mom, int(ierr)


def run_catalogue(xp, vp, mp, np_halo, nhalo, L_Box, link, np_halo_min, bound_check, verbose,
                  softening, a_val, b_val, s_15_val, n_threads, total_np, ng_val=256,
                  ng_global_val=512.0, slot=None, units=None):
    """run() plus the halo catalogue built on the device.  Returns
    (in_halo, halo_id, ang_mom, ierr, members, offsets): members (int32)
    lists each valid halo's particle indices, ascending, halos in id order;
    offsets[h]:offsets[h+1] delimits halo h+1."""
    L = load()
    n = int(total_np)
    if xp.flags.c_contiguous:
        layout = LAYOUT_SOA
    elif xp.flags.f_contiguous:
        layout = LAYOUT_AOS
    else:
        xp = np.ascontiguousarray(xp)
        layout = LAYOUT_SOA
    if vp is not None:
        vp = np.asarray(vp, dtype=np.float64)
        vp = np.ascontiguousarray(vp) if layout == LAYOUT_SOA else np.asfortranarray(vp)
    if mp is not None:
        mp = np.ascontiguousarray(mp, dtype=np.float64)
    nph = np.ascontiguousarray(np_halo, dtype=np.int32)
    halo_id = np.empty(n, dtype=np.int32)
    ang_mom = np.zeros((3, max(int(nhalo), 0)), dtype=np.float64, order="F")
    members = np.empty(max(n, 1), dtype=np.int32)
    cap = n // max(1, int(np_halo_min)) + 2
    offsets = np.empty(cap, dtype=np.int64)
    nfound = ctypes.c_int32(0)
    ierr = L.pyfof_run_catalogue(
        ctypes.c_void_p(slot) if slot else None, _units_ptr(units), _ptr(xp), _ptr(vp), _ptr(mp), layout,
        nph.ctypes.data_as(_i32p), int(nhalo), n, float(L_Box), float(link), int(np_halo_min),
        int(bound_check), int(verbose), float(softening), float(a_val), float(b_val), float(s_15_val),
        int(n_threads), int(ng_val), float(ng_global_val), _ptr(halo_id), ang_mom.ctypes.data_as(_dp),
        _ptr(members), _ptr(offsets), cap, ctypes.byref(nfound))
    k = int(nfound.value) if ierr == 0 else 0
    offsets = offsets[:k + 1] if k else np.zeros(1, dtype=np.int64)
    return halo_id > 0, halo_id, ang_mom, int(ierr), members[:int(offsets[-1])], offsets


def slot_create(device=0, pm_budget_bytes=0):
    """A slot of its own on `device` (calls on different slots overlap on
    the GPU).  Returns the handle (an int)."""
    h = ctypes.c_void_p()
    if load().pyfof_slot_create(int(device), int(pm_budget_bytes), ctypes.byref(h)) != 0:
        raise RuntimeError(last_error())
    return h.value


def slot_destroy(slot):
    if load().pyfof_slot_destroy(ctypes.c_void_p(slot)) != 0:
        raise RuntimeError(last_error())


def slot_stat(slot, key):
    v = ctypes.c_int64(0)
    if load().pyfof_slot_stat(ctypes.c_void_p(slot), key.encode(), ctypes.byref(v)) != 0:
        raise ValueError(last_error())
    return int(v.value)


def halo_potential(q, w, softening=0.1, a_val=1.0, s15=17.152, ng=256, fp64=False):
    """First-pass potential of one candidate (q: (3,np) positions relative to
    member 0, stable-id order).  Returns (phi float32, method gid)."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    n = w.shape[0]
    phi = np.zeros(n, np.float32)
    meth = ctypes.c_int32(-1)
    ierr = load().pyfof_halo_potential(q.ctypes.data, w.ctypes.data, n, float(softening),
                                       float(a_val), float(s15), int(ng), int(bool(fp64)),
                                       phi.ctypes.data, ctypes.byref(meth))
    if ierr:
        raise RuntimeError(f"ierr={ierr}: {last_error()}")
    return phi, int(meth.value)


def halo_potential_direct_static(q, w, softening=0.1, a_val=1.0, fp64=False, stream=0):
    """Direct-summation potential (np <= 1000) computed without any device
    allocation: scratch lives in the library's static device array.
    Returns (phi float32, ierr)."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    n = w.shape[0]
    phi = np.zeros(n, np.float32)
    ierr = load().pyfof_halo_potential_direct_static(
        q.ctypes.data, w.ctypes.data, n, float(softening), float(a_val), int(bool(fp64)),
        phi.ctypes.data, ctypes.c_void_p(stream) if stream else None)
    return phi, int(ierr)


def run_device(xp_ptr, vp_ptr, mp_ptr, layout, np_halo, nhalo, total_np, L_Box, link,
               np_halo_min, bound_check, verbose, softening, a_val, b_val, s_15_val, n_threads,
               in_halo_ptr, halo_id_ptr, ng_val=256, ng_global_val=512.0):
    """Device-memory call: pointers are integers (e.g. torch ``data_ptr()``).
    Returns (ang_mom, ierr)."""
    L = load()
    nph = np.ascontiguousarray(np_halo, dtype=np.int32)
    ang_mom = np.zeros((3, max(int(nhalo), 0)), dtype=np.float64, order="F")
    vp_c = ctypes.c_void_p(vp_ptr) if vp_ptr else None
    mp_c = ctypes.c_void_p(mp_ptr) if mp_ptr else None
    ierr = L.pyfof_run_device(ctypes.c_void_p(xp_ptr), vp_c, mp_c, int(layout),
                              nph.ctypes.data_as(_i32p), int(nhalo), int(total_np),
                              float(L_Box), float(link), int(np_halo_min), int(bound_check),
                              int(verbose), float(softening), float(a_val), float(b_val),
                              float(s_15_val), int(n_threads), int(ng_val), float(ng_global_val),
                              ctypes.c_void_p(in_halo_ptr), ctypes.c_void_p(halo_id_ptr),
                              ang_mom.ctypes.data_as(_dp))
    return ang_mom, int(ierr)
