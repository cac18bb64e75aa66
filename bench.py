#!/usr/bin/env python
"""Benchmark of the py_fof B200 hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload fof_unbind_256|fof_unbind_128|fof_256|fof_128|fof_64|
                                unbind_nfw_20k|unbind_nfw_2k]

One step = one full ``fof()`` call over one synthetic particle set.  The
default workload is FoF + unbinding (bound_check=True, cube units,
softening 0.1) on 256^3 = 16,777,216 particles in a periodic box of side 256:
70% uniform background, 30% in 4096 Plummer spheres (a = 1.5, member counts
dN/dM ~ M^-1.9 over 20..5000), lognormal masses (sigma_ln 0.3, mean 1),
virial velocities + bulk sigma 3 with 10% of members kicked by 3 sigma,
background sigma 1; link 0.2, np_halo_min 10, s_15 = 15 * 0.67 * 256 / 300.

* value: particles per second (Mpart/s) of the whole call (binning, linking,
  labelling, candidate packing, unbinding of every candidate, outputs) with
  the inputs resident in HBM, on the library's default FP64 unbinding path
  (the plain FP64 GPU path the FoF + unbinding configuration names),
  device-timed with CUDA events on the stream the library launches on.
  All ranks run their own replica (one periodic box is one region, which
  this path does not split): value = N * particles / max-over-ranks time.
* unbind: candidates unbound per second of unbinding stage time for the
  batched FP64 path (the value's), the batched FP32 product path and the
  plain per-halo FP64 path (one halo per launch sequence), each on the same
  input.
* e2e: the same metric through the public API ``py_fof_b200.fof`` with
  pinned host inputs, host<->device copies inside the timed region.
* roofline: the dominant kernel group.  With unbinding: the particle-mesh
  convolutions (the FFT kernels), algorithmic bytes 4 s (n+2) n^2 per solve
  on an n^3 grid of s-byte reals over their event-timed device time.  Plain
  FoF: the linking kernels, 20 B per particle + 4 B per cell.
  roofline_fof_link: the linking kernels on every workload.
* cpu_baseline: the CPU restatement of the reference (oracle/, OpenMP, the
  reference's thread policy) on this host: one full call of the workload
  after one untimed call on a sub-volume (which builds the Green tables),
  or, for workloads too large for one call in 30 s, a stated sample.
* --impl reference: the same restatement on the same workload, every timed
  step one full call; the untimed warm-up steps run on the sub-volume.
Under torchrun (N > 1) rank 0 prints the single JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Plummer boxes: name -> (n_side, bound_check); box side n_side, 4096
# (n_side/256)^3 halos.  NFW lists: name -> (halos, largest halo).
WORKLOADS = {
    "fof_unbind_256": ("box", 256, True),
    "fof_unbind_128": ("box", 128, True),
    "fof_256": ("box", 256, False),
    "fof_128": ("box", 128, False),
    "fof_64": ("box", 64, False),
    "unbind_nfw_20k": ("nfw", 20000, 2_000_000),
    "unbind_nfw_2k": ("nfw", 2000, 200_000),
    # lognormal field boxes: name -> (n_side, mesh); L = n_side, np_halo_min 20
    "fof_lognormal_1024": ("lognormal", 1024, 512),
    "fof_lognormal_512": ("lognormal", 512, 256),
    "fof_lognormal_256": ("lognormal", 256, 128),
    "fof_lognormal_128": ("lognormal", 128, 64),
}
# Warm-up input of the CPU arms (a sub-volume with the same recipe and
# density, or the first halos of the same list), and the CPU sample of the
# workloads too large for full CPU calls within the bench's time (None: the
# timed CPU calls run the workload itself)
CPU_WARMUP = {
    "fof_unbind_256": "fof_unbind_128",
    "fof_unbind_128": "fof_unbind_128",
    "fof_256": "fof_64",
    "fof_128": "fof_64",
    "fof_64": "fof_64",
    "unbind_nfw_20k": "unbind_nfw_20k:300",
    "unbind_nfw_2k": "unbind_nfw_2k:300",
    "fof_lognormal_1024": "fof_lognormal_128",
    "fof_lognormal_512": "fof_lognormal_128",
    "fof_lognormal_256": "fof_lognormal_128",
    "fof_lognormal_128": "fof_lognormal_128",
}
CPU_SAMPLE = {
    "unbind_nfw_20k": "unbind_nfw_20k:2000",
    "fof_lognormal_1024": "fof_lognormal_256",
    "fof_lognormal_512": "fof_lognormal_256",
}
LINK = 0.2
NP_MIN = 10
SOFTENING = 0.1
# algorithmic bytes of the linking kernel: 12 B position read, 4 B parent
# read, 4 B parent write per particle plus a 4 B cell offset per cell
LINK_BYTES_PER_PARTICLE = 20
LINK_BYTES_PER_CELL = 4


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _tile_table_note():
    """The tile table the library loaded (path relative to the repository and
    a hash of its contents), or the built-in defaults."""
    import hashlib
    from py_fof_b200 import _native
    p = _native.tile_table_used()
    if not p:
        return {"table": "built-in defaults"}
    return {"table": os.path.relpath(p, ROOT),
            "sha256_16": hashlib.sha256(open(p, "rb").read()).hexdigest()[:16]}


def _traffic(workload, kernel):
    """DRAM bytes per algorithmic byte of `kernel`, from a committed ncu
    summary (profiles/roofline_traffic.json), or None."""
    tp = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(tp):
        return None
    d = json.load(open(tp)).get(kernel)
    if not d:
        return None
    return float(d["dram_bytes_per_algorithmic_byte"])


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(name, seed=0, device=None):
    """Synthetic input of a workload: dict(xp (3,N), vp, mp (None = unit
    masses), np_halo, L, bound, s15, np_min, regions (the per-region arrays
    of a list input, else None)).  "name:K" keeps the first K regions of a
    list.  Lognormal boxes above 128^3 are generated on `device` (xp is then
    a torch tensor there)."""
    from py_fof_b200 import workloads as W
    base, _, keep = name.partition(":")
    kind, a, b = WORKLOADS[base]
    if kind == "lognormal":
        side, mesh = a, b
        dev = device if side > 128 else None
        xp = W.lognormal_box(side ** 3, float(side), mesh, seed=seed, device=dev)
        return dict(xp=xp, vp=None, mp=None, np_halo=[side ** 3], L=float(side), bound=False,
                    s15=15.0 * 0.67 * side / 300.0, ng_global=float(side), regions=None, np_min=20,
                    on_device=dev is not None)
    if kind == "box":
        side, bound = a, b
        halos = max(1, int(round(4096 * (side / 256.0) ** 3)))
        d = W.plummer_box(side ** 3, float(side), halos, seed=seed, with_velocities=bound,
                          lognormal_mass=0.3 if bound else None)
        # a sub-volume keeps the 256-box s_15 (the same physical scales)
        return dict(xp=d["xp"], vp=d["vp"], mp=d["mp"], np_halo=[side ** 3], L=float(side),
                    bound=bound, s15=15.0 * 0.67 * 256.0 / 300.0, ng_global=256.0, regions=None,
                    np_min=NP_MIN, on_device=False)
    xs, vs = W.nfw_halos(a, seed=seed, mmax=b)
    if keep:
        xs, vs = xs[:int(keep)], vs[:int(keep)]
    return dict(xp=np.ascontiguousarray(np.hstack(xs)), vp=np.ascontiguousarray(np.hstack(vs)), mp=None,
                np_halo=[x.shape[1] for x in xs], L=512.0, bound=True,
                s15=15.0 * 0.67 * 512.0 / 300.0, ng_global=512.0, regions=(xs, vs), np_min=NP_MIN,
                on_device=False)


def _config(workload, wl, n_job, world, scaling):
    """The config dict both arms print for one workload (the reference arm
    with world = 1)."""
    n = wl["xp"].shape[1]
    in_bytes = 24 * n + (24 * n if wl["vp"] is not None else 0) + (8 * n if wl["mp"] is not None else 0)
    l2 = (f"inputs larger than L2 ({in_bytes / 1e6:.0f} MB of positions, velocities and masses "
          "> 126 MB), no flush") if in_bytes > 126e6 else "inputs smaller than L2"
    return {"workload": workload, "particles": n_job if scaling == "strong" else n,
            "L_Box": wl["L"], "link": LINK, "np_halo_min": wl["np_min"], "bound_check": wl["bound"],
            "softening": SOFTENING, "s_15": wl["s15"], "regions": len(wl["np_halo"]),
            "unbinding": "fp64" if wl["bound"] else None, "l2": l2,
            "parallelism": (f"regions sharded x{world}" if scaling == "strong" else f"replicas x{world}")}


def cpu_port_run(wl, threads):
    """One call of the CPU restatement (oracle/) on the workload."""
    from oracle import oracle as O
    xp = np.asfortranarray(wl["xp"])
    n = xp.shape[1]
    vp = np.asfortranarray(wl["vp"]) if wl["vp"] is not None else np.zeros((3, n), order="F")
    mp = wl["mp"] if wl["mp"] is not None else np.ones(n)
    nph = np.asarray(wl["np_halo"], np.int32)
    t0 = time.perf_counter()
    _, hid, _, ierr = O.fof_fortran(xp, vp, mp, nph, len(nph), wl["L"], LINK, wl["np_min"],
                                    int(wl["bound"]), 0, SOFTENING, 1.0, 0.0, wl["s15"], threads, n)
    dt = time.perf_counter() - t0
    if ierr:
        raise RuntimeError(f"oracle ierr={ierr}")
    return dt, int(hid.max()), O.last_threads()


def _sample_kind(name, workload):
    if name == workload:
        return f"the {workload} workload itself"
    if ":" in name:
        return f"the first {name.partition(':')[2]} halos of the {workload} list"
    return f"a sub-volume of {workload} with the same recipe and density"


def _cpu_input(workload, seed):
    name = CPU_SAMPLE.get(workload, workload)
    return name, make_workload(name, seed)


def cpu_baseline(workload, seed):
    """The oracle on the workload (or its stated sample): one untimed call
    on the warm-up sub-volume (thread pool, Green tables), then one timed
    call."""
    threads = os.cpu_count() or 1
    cpu_port_run(make_workload(CPU_WARMUP[workload], seed), threads)
    name, wl = _cpu_input(workload, seed)
    dt, _, used = cpu_port_run(wl, threads)
    n = wl["xp"].shape[1]
    return {"value": n / dt / 1e6, "unit": "Mpart/s", "cores": used, "kind": "port",
            "sample": f"{name}: {n} particles, {_sample_kind(name, workload)}, one call after one "
                      f"untimed call on {CPU_WARMUP[workload]}, reference thread policy "
                      "(one region: 2 linking threads; unbinding in the reference's grid-class "
                      "groups, cost-ordered queues and phase/team split)"}


def run_reference(args):
    """--impl reference: the reference's CPU algorithm (restated in oracle/,
    the reference itself cannot be built here) with the reference's thread
    policy on all host cores.  Warm-up steps run on the workload's
    sub-volume; every timed step is one full call on the workload itself
    (or its stated sample for the two largest workloads)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    warm = make_workload(CPU_WARMUP[args.workload], args.seed)
    for _ in range(max(1, args.warmup)):
        cpu_port_run(warm, threads)
    del warm
    name, wl = _cpu_input(args.workload, args.seed)
    n = wl["xp"].shape[1]
    times, used = [], threads
    for _ in range(args.steps):
        dt, _, used = cpu_port_run(wl, threads)
        times.append(dt)
    t = sum(times) / len(times)
    v = n / t / 1e6
    line = {
        "impl": "reference", "metric": "fof_mpart_per_s", "value": v, "unit": "Mpart/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(args.workload, wl, n, 1, "weak"),
        "cpu_baseline": {"value": v, "unit": "Mpart/s", "cores": used, "kind": "port",
                         "sample": f"{name}: {n} particles per step, "
                                   f"{_sample_kind(name, args.workload)}; warm-up steps on "
                                   f"{CPU_WARMUP[args.workload]}; reference thread policy"},
        "e2e": {"value": v, "unit": "Mpart/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _exact_potential(q, w, targets, softening, a_val=1.0):
    """Exact softened direct-sum potential in FP64 (torch on the device, a
    plain library reference): phi_t = -a/(6 pi) sum_{j != t} w_j D(|q_j - q_t|)
    with D the spline-softened 1/r of the reference's direct path
    (bound_fortran.f90:3080-3102)."""
    import torch
    dev = torch.device("cuda")
    qd = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float64)).to(dev)
    wd = torch.from_numpy(np.ascontiguousarray(w, dtype=np.float64)).to(dev)
    tg = torch.from_numpy(np.ascontiguousarray(targets, dtype=np.int64)).to(dev)
    h = float(softening)
    out = torch.empty(len(targets), dtype=torch.float64, device=dev)
    n = q.shape[1]
    step = max(1, (1 << 26) // max(n, 1))
    for s0 in range(0, len(targets), step):
        t = tg[s0:s0 + step]
        d = qd[:, None, :] - qd[:, t, None]
        r = torch.sqrt((d * d).sum(0))
        e = 2.0 * r / h
        inner = (208.0 - e * e * (112.0 + e * e * (-56.0 + e * (14.0 + e * (8.0 - 3.0 * e))))) / (70.0 * h)
        es = torch.clamp(e, min=1e-300)
        outer = (128.0 - (e * e * (448.0 + e * (-280.0 + e * (56.0 + e * (14.0 + e * (-8.0 + e)))))
                          - 224.0 * e - 12.0 / es)) / (70.0 * h)
        D = torch.where(r >= h, 1.0 / torch.clamp(r, min=1e-300), torch.where(e <= 1.0, inner, outer))
        D[torch.arange(len(t), device=dev), t] = 0.0  # no self term
        out[s0:s0 + len(t)] = -(a_val / (6.0 * np.pi)) * (D * wd[None, :]).sum(1)
    return out.cpu().numpy()


def potential_error_report(d, seed=0, per_stratum=6):
    """Per-halo first-pass potential errors of the FP32 product path against
    the FP64 device path and both against the exact FP64 direct sum, and the
    energy error of each halo's final kept set (FP32 path), for a sample of
    the list's halos stratified by size.  Errors are max |phi - phi_ref| over
    the compared members divided by max |phi_ref| of the halo; energies are
    specific energies 1/2 |v - v_c|^2 + phi of the kept members (v_c their
    mean velocity) with the FP32 path's and the exact potential of the kept
    set, divided by max |E|.  Halos above 20,000 members are compared at
    4096 sampled members."""
    import py_fof_b200 as P
    from py_fof_b200 import _native
    xs, vs = d["regions"]
    sizes = np.array([x.shape[1] for x in xs])
    strata = [("direct", 0, 1000), ("pm_1k_5k", 1000, 5000), ("pm_5k_20k", 5000, 20000),
              ("pm_20k_200k", 20000, 200000), ("pm_200k_up", 200000, 1 << 40)]
    rng = np.random.default_rng(seed + 77)
    kw = dict(vp_list=vs, L_Box=d["L"], linking_length=LINK, np_halo_min=d["np_min"], bound_check=True,
              softening=SOFTENING, ng_global=d["ng_global"])
    with _native.options(unbind_fp64=0):
        ih32 = P.fof(xs, **kw)
    off = np.concatenate([[0], np.cumsum(sizes)])
    out = {}
    for name, lo, hi in strata:
        idx = np.nonzero((sizes > lo) & (sizes <= hi))[0]
        if idx.size == 0:
            continue
        pick = rng.choice(idx, size=min(per_stratum, idx.size), replace=False)
        rows = []
        for r in pick:
            x, v = xs[r], vs[r]
            n = x.shape[1]
            q = (x - x[:, :1]).astype(np.float32)
            w = np.ones(n, np.float32)
            p32, g = _native.halo_potential(q, w, softening=SOFTENING, s15=d["s15"], fp64=False)
            p64, _ = _native.halo_potential(q, w, softening=SOFTENING, s15=d["s15"], fp64=True)
            tg = np.arange(n) if n <= 20000 else np.sort(rng.choice(n, 4096, replace=False))
            ex = _exact_potential(q, w, tg, SOFTENING)
            sc = np.abs(ex).max()
            row = {"np": int(n), "method": int(g),
                   "fp32_vs_fp64": float(np.abs(p32 - p64).max() / np.abs(p64).max()),
                   "fp32_vs_exact": float(np.abs(p32[tg] - ex).max() / sc),
                   "fp64_vs_exact": float(np.abs(p64[tg] - ex).max() / sc)}
            keep = np.nonzero(ih32[off[r]:off[r] + n])[0]
            if keep.size >= 2:
                qk = (x[:, keep] - x[:, keep[:1]]).astype(np.float32)
                wk = np.ones(keep.size, np.float32)
                pk32, _ = _native.halo_potential(qk, wk, softening=SOFTENING, s15=d["s15"], fp64=False)
                tk = np.arange(keep.size) if keep.size <= 20000 else \
                    np.sort(rng.choice(keep.size, 4096, replace=False))
                exk = _exact_potential(qk, wk, tk, SOFTENING)
                vk = v[:, keep] - v[:, keep].mean(axis=1, keepdims=True)
                kin = 0.5 * (vk[:, tk] ** 2).sum(0)
                e_ex = kin + exk
                row["kept"] = int(keep.size)
                row["energy_fp32_vs_exact"] = float(np.abs((kin + pk32[tk]) - e_ex).max() /
                                                    np.abs(e_ex).max())
            rows.append(row)
        summ = {"halos": len(rows), "np_range": [int(min(r["np"] for r in rows)),
                                                 int(max(r["np"] for r in rows))]}
        for key in ("fp32_vs_fp64", "fp32_vs_exact", "fp64_vs_exact", "energy_fp32_vs_exact"):
            vals = np.array([r[key] for r in rows if key in r])
            if vals.size:
                summ[key] = {"p50": float(np.percentile(vals, 50)), "p99": float(np.percentile(vals, 99)),
                             "max": float(vals.max())}
        out[name] = summ
    return out


def run_b200(args):
    import torch
    import torch.distributed as dist

    import py_fof_b200 as P
    from py_fof_b200 import _native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    L_ = _native.load()
    if L_.pyfof_init(local) != 0:
        raise RuntimeError(_native.last_error())
    dev = torch.device("cuda", local)
    d = make_workload(args.workload, args.seed, device=dev)
    if d["on_device"]:
        torch.cuda.empty_cache()  # the generator's temporaries go back to the driver
    Lbox, bound, s15 = d["L"], d["bound"], d["s15"]
    nph = list(d["np_halo"])
    n = d["xp"].shape[1]
    n_job = world * n  # particles of the whole job: N replicas of a box
    scaling = "weak"
    if world > 1 and d["regions"] is not None:
        # a list input is split into contiguous blocks of regions, one per rank
        from py_fof_b200.shard import partition_regions
        s_r, e_r = partition_regions(nph, world, bound)[rank]
        off = np.concatenate([[0], np.cumsum(nph)]).astype(np.int64)
        sl = slice(int(off[s_r]), int(off[e_r]))
        xs, vs = d["regions"]
        d = dict(d, xp=np.ascontiguousarray(d["xp"][:, sl]),
                 vp=np.ascontiguousarray(d["vp"][:, sl]) if d["vp"] is not None else None,
                 mp=d["mp"][sl] if d["mp"] is not None else None,
                 np_halo=nph[s_r:e_r], regions=(xs[s_r:e_r], vs[s_r:e_r]))
        n_job = n
        nph = list(d["np_halo"])
        n = d["xp"].shape[1]
        scaling = "strong"
    dev = torch.device("cuda", local)
    xp = d["xp"] if d["on_device"] else torch.from_numpy(d["xp"]).to(dev)
    vp = torch.from_numpy(d["vp"]).to(dev) if d["vp"] is not None else None
    mp = torch.from_numpy(d["mp"]).to(dev) if d["mp"] is not None else None
    ih = torch.zeros(n, dtype=torch.int32, device=dev)
    hid = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    _native.set_stream(stream.cuda_stream)

    def step():
        _, ierr = _native.run_device(
            xp.data_ptr(), vp.data_ptr() if vp is not None else 0,
            mp.data_ptr() if mp is not None else 0, _native.LAYOUT_SOA, nph, len(nph), n, Lbox, LINK,
            d["np_min"], int(bound), 0, SOFTENING, 1.0, 0.0, s15, 0, ih.data_ptr(), hid.data_ptr())
        if ierr:
            raise RuntimeError(f"ierr={ierr}: {_native.last_error()}")

    def timed(steps):
        """Device time per call over `steps` back-to-back calls (no stage
        timers, no host reads between calls)."""
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    def stages(k=2):
        """Stage device times (library timers) averaged over k more calls,
        outside any timed region."""
        st = []
        with _native.options(timing=1):
            for _ in range(k):
                step()
                st.append({key: _native.last_stage_ms(key) for key in ("link", "fof", "unbind", "call",
                                                                        "pm_fft")}
                          | {"pm_fft_bytes": _native.get_stat("pm_fft_bytes")})
        return {key: sum(x[key] for x in st) / len(st) for key in st[0]}

    # the product path: the library default (FP64 unbinding); --fp32 selects
    # the FP32 path for profiler runs
    if args.profile_run and args.fp32:
        _native.set_option("unbind_fp64", 0)
    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize(dev)
    launches0 = _native.get_stat("launches")
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ms = timed(args.steps)
    clocks = sampler.stop()
    launches = _native.get_stat("launches") - launches0
    if world > 1:
        dist.barrier()
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = n_job / (ms_max * 1e-3) / 1e6
    ngroups = int(hid.max().item())
    counts = {k: _native.get_stat(k) for k in ("candidates", "direct_halos", "pm_halos",
                                               "valid_halos", "pm_solves")}
    ncells = _native.get_stat("cells")
    st = stages()

    if args.profile_run:
        # only the warm-up and timed product steps (for a profiler's launch list)
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"profile_run": args.workload, "ms_per_step": ms_max,
                              "gpu_launches": launches, "pm_fft_bytes_per_call": st["pm_fft_bytes"],
                              "pm_fft_ms_per_call": st["pm_fft"], "pm_solves": counts["pm_solves"],
                              "link_ms": st["link"], "cells": ncells}),
                  flush=True)
        return 0

    unbind = None
    fp32_st = None
    if bound:
        ncand = counts["candidates"]

        def leg(ms_call, st_):
            u = st_["unbind"]
            return {"halos_per_s": ncand / (u * 1e-3) if u > 0 else None, "unbind_ms": u,
                    "call_ms": ms_call}

        legs = {"fp64_batched": leg(ms, st)}
        with _native.options(unbind_fp64=0):
            step()
            ms32 = timed(max(1, args.steps // 3))
            fp32_st = stages()
            legs["fp32_batched"] = leg(ms32, fp32_st)
        with _native.options(unbind_per_halo=1):
            ms_ph = timed(1)
            legs["fp64_per_halo"] = leg(ms_ph, stages(1))
        base = legs["fp64_per_halo"]["halos_per_s"]
        unbind = {"halos": ncand, "direct": counts["direct_halos"], "pm": counts["pm_halos"],
                  "valid": counts["valid_halos"], "pm_solves": counts["pm_solves"], **legs,
                  "fp32_vs_fp64_per_halo": (legs["fp32_batched"]["halos_per_s"] / base) if base else None,
                  "fp32_vs_fp64_batched": (legs["fp32_batched"]["halos_per_s"] /
                                           legs["fp64_batched"]["halos_per_s"])}
        if d["regions"] is not None and rank == 0 and not args.no_errors:
            unbind["errors"] = potential_error_report(d, args.seed)

    # end to end through the public API with pinned host buffers
    def pinned(a):
        if a is None:
            return None
        p = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        p.copy_(torch.from_numpy(a))
        return p.numpy()

    e2e_note = None
    if d["on_device"] and 24 * n > (8 << 30):
        # a host copy of the input would exceed what the host can pin
        e2e_value, h2d, d2h = None, 0, 0
        e2e_note = f"not measured: {24 * n / 1e9:.1f} GB of positions generated on the device"
    else:
        if d["on_device"]:
            xp_h = torch.empty(tuple(xp.shape), dtype=torch.float64, pin_memory=True)
            xp_h.copy_(xp)
            xp_h, vp_h, mp_h = xp_h.numpy(), None, None
        elif d["regions"] is None:
            xp_h, vp_h, mp_h = pinned(d["xp"]), pinned(d["vp"]), pinned(d["mp"])
        else:  # list input, as the reference API takes it
            xp_h, vp_h, mp_h = list(d["regions"][0]), list(d["regions"][1]), None
        _native.set_stream(0)
        kw = dict(vp_list=vp_h, mp_list=mp_h, L_Box=Lbox, linking_length=LINK, np_halo_min=d["np_min"],
                  bound_check=bound, softening=SOFTENING, ng_global=d["ng_global"])
        for _ in range(max(1, min(args.warmup, 2))):
            P.fof(xp_h, **kw)
        e2e_t = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            P.fof(xp_h, **kw)
            e2e_t.append(time.perf_counter() - t0)
        e2e_s = torch.tensor([sum(e2e_t) / len(e2e_t)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
        e2e_value = n_job / float(e2e_s.item()) / 1e6
        h2d = 24 * n + (24 * n if vp_h is not None else 0) + (8 * n if mp_h is not None else 0)
        # in_halo (one byte per particle: fof() returns no halo ids) and ang_mom
        d2h = n + 24 * (len(d["regions"][0]) if d["regions"] is not None else 1)

    peak, peak_kind = _peaks()

    def roof(kname, k_ms, k_bytes, extra):
        achieved = k_bytes / (k_ms * 1e-3) / 1e9 if k_ms > 0 else None
        ratio = _traffic(args.workload, kname)
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": ratio * k_bytes if ratio is not None else None,
                "kernel": kname, "peak_kind": peak_kind, "algorithmic_bytes_per_call": k_bytes,
                "kernel_ms_per_call": k_ms, **extra}

    link_bytes = LINK_BYTES_PER_PARTICLE * n + LINK_BYTES_PER_CELL * ncells
    roof_link = roof("fof_link", st["link"], link_bytes,
                     {"kernels": "fof_link_dense_kernel + fof_link_kernel (one link stage)",
                      "algorithmic_bytes": "20 B per particle + 4 B per cell"})
    if bound:
        roof_main = roof("pm_convolve_fp64", st["pm_fft"], st["pm_fft_bytes"],
                         {"kernels": "k_x_r2c, k_lines (3 launches), k_x_c2r per batch (FP64 grids)",
                          "algorithmic_bytes": "32 (n+2) n^2 per solve on FP64 grids (a read and a "
                                               "write of the padded grid per transform, two transforms)",
                          "solves_per_call": counts["pm_solves"]})
    else:
        roof_main = roof_link

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.workload, args.seed)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "fof_mpart_per_s", "value": value, "unit": "Mpart/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "higher_is_better": True, "scaling": scaling, "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": _config(args.workload, d, n_job, world, scaling),
        "groups": ngroups,
        "stages_ms": {"fof": st["fof"], "link_kernel": st["link"], "unbind": st["unbind"],
                      "pm_fft": st["pm_fft"]},
        "unbind": unbind,
        "e2e": {"value": e2e_value, "unit": "Mpart/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, **({"note": e2e_note} if e2e_note else {})},
        "roofline": roof_main,
        "roofline_fof_link": roof_link,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "tile_table": _tile_table_note(),
    }
    print(json.dumps(line), flush=True)
    return 0


SERVE_REQUESTS = 2000
SERVE_LOG_RANGE = (4.0, 8.0)


def serve_pool(seed=0, count=24, log_range=SERVE_LOG_RANGE):
    """Distinct requests of the serving configuration: sizes log-uniform on
    [1e4, 1e8] particles, the 64^3 recipe scaled to L_Box = N^(1/3) (64
    halos per 262,144 particles); every second request with unbinding
    (lognormal masses), half of those in physical units; ng_global = 512
    keeps s_15 above the candidate spans.  The stream draws its requests
    from this pool."""
    from py_fof_b200 import workloads as W
    rng = np.random.default_rng(seed)
    pool = []
    for k in range(count):
        n = int(10 ** rng.uniform(*log_range))
        L = float(n ** (1.0 / 3.0))
        bound = k % 2 == 1
        d = W.plummer_box(n, L, max(1, round(64 * n / 262144)), seed=seed * 1000 + k,
                          with_velocities=bound, lognormal_mass=0.3 if bound else None)
        kw = dict(L_Box=L, linking_length=LINK, np_halo_min=NP_MIN, ng_global=512.0)
        if bound:
            kw.update(vp_list=d["vp"], mp_list=d["mp"], bound_check=True, softening=SOFTENING)
            if k % 4 == 3:
                kw.update(units="physical", softening=0.05)
        pool.append((d["xp"], kw, n))
    return pool


def _serve_run(pool, order, arrivals, slots):
    """Submit pool[order[i]] at arrivals[i] (seconds from start); returns
    (latencies ms, makespan s, particles, max concurrent)."""
    from py_fof_b200 import serve
    srv = serve.Server(slots=slots)
    t0 = time.perf_counter()
    futs = []
    for i, k in enumerate(order):
        dt = t0 + arrivals[i] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        x, kw, _ = pool[k]
        futs.append(srv.submit(x, **kw))
    for f in futs:
        f.result()
    t1 = time.perf_counter()
    lat = srv.latencies_ms()
    most = srv.max_running
    srv.close()
    return lat, t1 - t0, sum(pool[k][2] for k in order), most


def run_serve(args):
    """--workload serve: requests with Poisson arrivals, served by the
    continuous-batching loop (4 slots) and, on the same arrival times, one at
    a time (1 slot); p50/p99 latency and throughput of both."""
    import torch
    import py_fof_b200 as P
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pool = serve_pool(args.seed)
    # calibration: every pool request alone (also builds the Green tables)
    for x, kw, _ in pool:
        P.fof_with_info(x, **kw)
    svc = []
    for x, kw, _ in pool:
        t = time.perf_counter()
        P.fof_with_info(x, **kw)
        svc.append(time.perf_counter() - t)
    rate = 1.25 / float(np.mean(svc))  # offered load: 1.25x one-at-a-time capacity
    nreq = SERVE_REQUESTS
    rng = np.random.default_rng(args.seed + 1)
    order = rng.integers(0, len(pool), nreq)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    res = {}
    for name, slots in (("one_at_a_time", 1), ("served", 4)):
        lat, span, parts, most = _serve_run(pool, order, arrivals, slots)
        res[name] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "req_per_s": nreq / span, "mpart_per_s": parts / span / 1e6, "slots": slots,
                     "max_concurrent": most}
    if rank != 0:
        return 0
    s = res["served"]
    h2d = float(np.mean([24 * n * (2 if "vp_list" in kw else 1) + (8 * n if "mp_list" in kw else 0)
                         for _, kw, n in (pool[k] for k in order)]))
    line = {
        "metric": "serve_mpart_per_s", "value": s["mpart_per_s"], "unit": "Mpart/s",
        "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": 1e3 / s["req_per_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "serve", "requests": nreq, "distinct_inputs": len(pool),
                   "sizes": "log-uniform 1e4..1e8", "offered_req_per_s": rate,
                   "arrivals": "Poisson", "unbinding_share": 0.5},
        "serve": res,
        "e2e": {"value": s["mpart_per_s"], "unit": "Mpart/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": float(np.mean([8 * pool[k][2] for k in order]))},
        "service_alone_ms": {"mean": 1e3 * float(np.mean(svc)), "max": 1e3 * float(np.max(svc))},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fof_unbind_256", choices=sorted(WORKLOADS) + ["serve"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-errors", action="store_true",
                    help="skip the per-halo potential error report of list workloads")
    ap.add_argument("--fp32", action="store_true",
                    help="with --profile-run: the FP32 unbinding path")
    ap.add_argument("--profile-run", action="store_true",
                    help="run only the warm-up and timed steps of the default path")
    args = ap.parse_args()
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop; "
                              "its per-request CPU cost is the cpu_baseline of the box workloads"}))
            return 0
        return run_serve(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
