#!/usr/bin/env python
"""Benchmark of the py_fof B200 hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload fof256|fof64|unbind256]

One step = one full ``fof()`` call (binning, linking, labelling, candidate
statistics; with --workload unbind256 also the unbinding of every candidate)
over one synthetic particle set.  Default workload: 256^3 = 16,777,216
particles in a periodic box of side 256 with 4096 Plummer halos (70% uniform
background), link 0.2, np_halo_min 10.

* value: particles per second (Mpart/s) with the inputs resident in HBM,
  device-timed with CUDA events on the stream the library launches on; all
  ranks run their own replica (the periodic box is one region, which this
  path does not split), value = N * particles / max-over-ranks time.
* e2e: the same metric through the public API ``py_fof_b200.fof`` with
  host (pinned) input arrays, host<->device copies inside the timed region.
* roofline: the linking kernel's algorithmic bytes per launch over its
  event-timed duration, against the measured HBM copy bandwidth.
* cpu_baseline: the CPU restatement of the reference (oracle/, OpenMP) timed
  on this host on the same workload.
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

WORKLOADS = {
    # name: (n_side, L, halos, bound_check)
    "fof256": (256, 256.0, 4096, False),
    "fof64": (64, 64.0, 64, False),
    "fof128": (128, 128.0, 512, False),
    "unbind256": (256, 256.0, 4096, True),
}
LINK = 0.2
NP_MIN = 10
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


def make_workload(name, seed=0):
    from py_fof_b200 import workloads as W
    n_side, L, halos, bound = WORKLOADS[name]
    d = W.plummer_box(n_side ** 3, L, halos, seed=seed, with_velocities=bound,
                      lognormal_mass=0.3 if bound else None)
    return d, L, bound


def cpu_port_run(d, L, bound, threads):
    """One call of the CPU restatement (oracle/) on the workload."""
    from oracle import oracle as O
    xp = np.asfortranarray(d["xp"])
    n = xp.shape[1]
    vp = np.asfortranarray(d["vp"]) if d["vp"] is not None else np.zeros((3, n), order="F")
    mp = d["mp"] if d["mp"] is not None else np.ones(n)
    t0 = time.perf_counter()
    _, hid, _, ierr = O.fof_fortran(xp, vp, mp, np.array([n], np.int32), 1, L, LINK, NP_MIN,
                                    int(bound), 0, 0.1, 1.0, 0.0, 15 * 0.67 * L / 300.0,
                                    threads, n)
    dt = time.perf_counter() - t0
    if ierr:
        raise RuntimeError(f"oracle ierr={ierr}")
    return dt, int(hid.max()), O.last_threads()


def run_reference(args):
    """--impl reference: the reference's CPU algorithm (restated in oracle/,
    no reference build is possible here) on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    d, L, bound = make_workload(args.workload, args.seed)
    n = d["xp"].shape[1]
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_port_run(d, L, bound, threads)
    times = []
    for _ in range(args.steps):
        dt, _, used = cpu_port_run(d, L, bound, threads)
        times.append(dt)
    t = sum(times) / len(times)
    v = n / t / 1e6
    line = {
        "impl": "reference", "metric": "fof_mpart_per_s", "value": v, "unit": "Mpart/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "L_Box": L, "link": LINK,
                   "np_halo_min": NP_MIN, "bound_check": bound},
        "cpu_baseline": {"value": v, "unit": "Mpart/s", "cores": used, "kind": "port",
                         "sample": f"full workload ({n} particles) per step, reference "
                                   "thread policy (one region: 2 linking threads)"},
        "e2e": {"value": v, "unit": "Mpart/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


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
    d, Lbox, bound = make_workload(args.workload, args.seed)
    n = d["xp"].shape[1]
    dev = torch.device("cuda", local)
    xp = torch.from_numpy(d["xp"]).to(dev)
    vp = torch.from_numpy(d["vp"]).to(dev) if d["vp"] is not None else None
    mp = torch.from_numpy(d["mp"]).to(dev) if d["mp"] is not None else None
    ih = torch.zeros(n, dtype=torch.int32, device=dev)
    hid = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    _native.set_stream(stream.cuda_stream)
    _native.set_option("timing", 1)
    s15 = 15.0 * 0.67 * Lbox / 300.0

    def step():
        am, ierr = _native.run_device(
            xp.data_ptr(), vp.data_ptr() if vp is not None else 0,
            mp.data_ptr() if mp is not None else 0, _native.LAYOUT_SOA, [n], 1, n, Lbox, LINK,
            NP_MIN, int(bound), 0, 0.1, 1.0, 0.0, s15, 0, ih.data_ptr(), hid.data_ptr())
        if ierr:
            raise RuntimeError(f"ierr={ierr}: {_native.last_error()}")
        return _native.last_link_ms()

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize(dev)
    launches0 = _native.get_stat("launches")
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t_start.record(stream)
    link_ms = []
    for _ in range(args.steps):
        link_ms.append(step())
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    launches = _native.get_stat("launches") - launches0
    if world > 1:
        dist.barrier()
    ms = t_start.elapsed_time(t_end) / args.steps
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * n / (ms_max * 1e-3) / 1e6
    ngroups = int(hid.max().item())

    # end to end through the public API with pinned host buffers
    xp_pin = torch.empty((3, n), dtype=torch.float64, pin_memory=True)
    xp_pin.copy_(torch.from_numpy(d["xp"]))
    xp_h = xp_pin.numpy()
    vp_h = None
    if d["vp"] is not None:
        vp_pin = torch.empty((3, n), dtype=torch.float64, pin_memory=True)
        vp_pin.copy_(torch.from_numpy(d["vp"]))
        vp_h = vp_pin.numpy()
    _native.set_stream(0)
    kw = dict(vp_list=vp_h, L_Box=Lbox, linking_length=LINK, np_halo_min=NP_MIN,
              bound_check=bound, mp_list=d["mp"])
    for _ in range(max(1, args.warmup)):
        P.fof(xp_h, **kw)
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        P.fof(xp_h, **kw)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_t) / len(e2e_t)
    e2e_t_all = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t_all, op=dist.ReduceOp.MAX)
    e2e_value = world * n / float(e2e_t_all.item()) / 1e6
    h2d = 24 * n + (24 * n if vp_h is not None else 0) + (8 * n if d["mp"] is not None else 0)
    d2h = 8 * n + 24

    # roofline of the linking kernel
    peak, peak_kind = _peaks()
    link_ms_avg = sum(link_ms) / len(link_ms)
    ncell = _native.get_stat("cells")
    link_bytes = LINK_BYTES_PER_PARTICLE * n + LINK_BYTES_PER_CELL * ncell
    achieved = link_bytes / (link_ms_avg * 1e-3) / 1e9 if link_ms_avg > 0 else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "link_traffic.json")
    if os.path.exists(tp):
        tj = json.load(open(tp))
        if tj.get("workload") == args.workload:
            traffic = tj.get("dram_bytes_per_launch")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sample_name = "fof64" if args.workload != "fof64" else "fof64"
        ds, Ls, bs = make_workload(sample_name, args.seed)
        threads = os.cpu_count() or 1
        cpu_port_run(ds, Ls, bs, threads)
        dts = []
        deadline = time.perf_counter() + 15.0
        while time.perf_counter() < deadline or not dts:
            dt, _, used = cpu_port_run(ds, Ls, bs, threads)
            dts.append(dt)
        ns = ds["xp"].shape[1]
        cpu = {"value": ns / (sum(dts) / len(dts)) / 1e6, "unit": "Mpart/s", "cores": used,
               "kind": "port",
               "sample": f"{sample_name}: {ns} particles, same recipe and density, "
                         f"{len(dts)} calls in ~15 s, reference thread policy"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "fof_mpart_per_s", "value": value, "unit": "Mpart/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "L_Box": Lbox, "link": LINK,
                   "np_halo_min": NP_MIN, "bound_check": bound, "groups": ngroups,
                   "l2": "inputs larger than L2 (402 MB positions)" if n >= 2 ** 24 else
                         "inputs smaller than L2",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "Mpart/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": "fof_link_kernel", "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": link_bytes, "kernel_ms": link_ms_avg},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fof256", choices=sorted(WORKLOADS))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
