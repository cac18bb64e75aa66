"""List inputs sharded across ranks (one process per GPU).

The regions of a list input are independent for both FoF and unbinding
(fof_fortran.f90:158-173: every region is linked, and its candidates unbound,
on its own), so a call splits into contiguous blocks of regions, one per
rank, with no exchange during the computation.  Afterwards the ranks
exchange their outputs: a rank's halo ids are shifted by the number of valid
halos of the ranks before it, which reproduces the single-call numbering
(valid halos numbered 1.. in region order, fof_fortran.f90:313-355), and the
particle and region arrays are concatenated in rank order.  Every rank
returns the full result.

Errors: the ranks exchange their outcome before the outputs; if any rank
failed, every rank raises the error of the lowest failing rank, which holds
the earliest regions — the error the single call reports first (the
reference classifies candidates in region order, first error wins).

The exchange uses torch.distributed (NCCL on GPUs, gloo on CPU); the
process group and its timeout belong to the caller.
"""
from __future__ import annotations

import numpy as np

__all__ = ["partition_regions", "fof_core_sharded", "fof_sharded", "fof_with_info_sharded"]


def partition_regions(np_halo, world, bound_check=False):
    """Contiguous blocks of regions, one per rank, balanced by an estimated
    cost: particles for FoF, particles x log2(particles) with unbinding (the
    large halos dominate, PM passes over grids that grow with them).
    Returns a list of (start, end) region ranges; a rank may get none."""
    nph = np.asarray(np_halo, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = nph * np.maximum(1.0, np.log2(np.maximum(nph, 2.0))) if bound_check else nph.copy()
    cost = np.maximum(cost, 1.0)  # every region has a fixed overhead
    csum = np.concatenate([[0.0], np.cumsum(cost)])
    total = csum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(csum, total * r / world, side="left")))
    cuts.append(len(nph))
    cuts = np.maximum.accumulate(np.minimum(cuts, len(nph)))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def _slice_per_region(v, start, end, nph, total):
    """The part of a per-particle or per-region argument that belongs to
    regions [start, end), in the forms _fof_core accepts."""
    if v is None or np.isscalar(v) or (isinstance(v, np.ndarray) and v.ndim == 0):
        return v
    if isinstance(v, (list, tuple)):
        return list(v[start:end])
    if isinstance(v, np.ndarray) and v.ndim == 1:
        if len(v) == total:
            off = np.concatenate([[0], np.cumsum(nph)])
            return v[off[start]:off[end]]
        if len(v) == len(nph):
            return v[start:end]
    raise ValueError("unsupported per-region argument for a sharded call")


def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("a sharded call needs an initialised torch.distributed process group")
    return dist


def _gather_var(arr, dtype, group, dev):
    """All-gather of 1-D arrays of different lengths; returns the list."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    t = torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype).to(dev)
    n = torch.tensor([t.numel()], dtype=torch.int64, device=dev)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    m = max(1, max(int(x.item()) for x in ns))
    pad = torch.zeros(m, dtype=dtype, device=dev)
    pad[:t.numel()] = t
    outs = [torch.empty(m, dtype=dtype, device=dev) for _ in range(world)]
    dist.all_gather(outs, pad, group=group)
    return [o[:int(k.item())].cpu().numpy() for o, k in zip(outs, ns)]


def fof_core_sharded(xp_list, vp_list=None, mp_list=None, group=None, core=None, **kw):
    """`_fof_core` over a list input split across the ranks of `group`.

    Returns (in_halo, halo_id, ang_mom) of the whole list on every rank,
    equal to the single-call result.  `core` computes one rank's share (the
    native `_fof_core` by default)."""
    import torch
    from . import _fof_core
    dist = _dist()
    core = core or _fof_core
    if isinstance(xp_list, np.ndarray):
        xp_list = [xp_list]
    xp_list = list(xp_list)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    nph = [int(x.shape[1]) for x in xp_list]
    total = sum(nph)
    s, e = partition_regions(nph, world, bool(kw.get("bound_check", False)))[rank]
    err = None
    ih = np.zeros(0, dtype=bool)
    hid = np.zeros(0, dtype=np.int32)
    am = np.zeros((3, 0), dtype=np.float64)
    if e > s:
        try:
            ih, hid, am = core(xp_list[s:e], vp_list=_slice_per_region(vp_list, s, e, nph, total),
                               mp_list=_slice_per_region(mp_list, s, e, nph, total), **kw)
        except (ValueError, RuntimeError) as exc:
            err = (type(exc).__name__, str(exc))
    outcomes = [None] * world
    dist.all_gather_object(outcomes, err, group=group)
    for o in outcomes:
        if o is not None:
            raise (ValueError if o[0] == "ValueError" else RuntimeError)(o[1])
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    ihs = _gather_var(np.asarray(ih, dtype=np.uint8), torch.uint8, group, dev)
    hids = _gather_var(np.asarray(hid, dtype=np.int32), torch.int32, group, dev)
    ams = _gather_var(np.asarray(am, dtype=np.float64).T.reshape(-1), torch.float64, group, dev)
    halo_id = []
    shift = 0
    for h in hids:
        h = h.astype(np.int32)
        halo_id.append(np.where(h > 0, h + shift, 0).astype(np.int32))
        shift += int(h.max()) if h.size else 0
    in_halo = np.concatenate(ihs).astype(bool) if ihs else np.zeros(0, bool)
    halo_id = np.concatenate(halo_id) if halo_id else np.zeros(0, np.int32)
    ang_mom = np.concatenate([a.reshape(-1, 3) for a in ams], axis=0).T.copy()
    return in_halo, halo_id, np.asfortranarray(ang_mom)


def fof_sharded(xp_list, return_ang_mom=False, group=None, **kw):
    """`fof` over a list input split across the ranks of `group`."""
    in_halo, _, ang_mom = fof_core_sharded(xp_list, group=group, return_ang_mom=return_ang_mom, **kw)
    return (in_halo, ang_mom) if return_ang_mom else in_halo


def fof_with_info_sharded(xp_list, return_ang_mom=False, group=None, **kw):
    """`fof_with_info` over a list input split across the ranks of `group`."""
    from . import catalogue_from_ids
    in_halo, halo_id, ang_mom = fof_core_sharded(xp_list, group=group, return_ang_mom=return_ang_mom, **kw)
    return catalogue_from_ids(in_halo, halo_id, ang_mom, return_ang_mom)
