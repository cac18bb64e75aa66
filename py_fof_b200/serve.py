"""Serving loop: many `fof_with_info` requests of mixed sizes on one GPU.

Requests are admitted continuously: a request starts as soon as a slot is
free and its device-memory estimate fits in the HBM budget next to the
requests already running, so work that arrives while others are on the GPU
joins them instead of waiting for the queue to drain.  Each slot is a native
context of its own (CUDA streams and scratch, `pyfof_slot_create`) driven by
one host thread; the native call releases the GIL, so the calls of different
slots overlap on the device — the short launch-bound stages of small
requests fill the gaps of the large ones.  Device scratch stays cached in the
stream-ordered pool between requests, and the Green's-function tables are
shared by all slots.

Admission order: first come, first served; a request that does not fit may
be passed by later requests that do, at most `max_bypass` times, after which
nothing is admitted until it fits.  A request larger than the whole budget
runs alone.  Memory estimates start from per-particle constants and follow
the largest per-particle peak the slots have reported.

Results are those of `py_fof_b200.fof_with_info` for the same arguments (the
same validation, unit conversion, error mapping and catalogue).
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import threading
import time

import numpy as np

from . import FofCall, _catalogue_call, _finish, _native, _prepare, catalogue_from_ids

__all__ = ["Server"]


class _Request:
    __slots__ = ("rid", "call", "ret_am", "future", "est", "arrival", "start", "end", "bypassed",
                 "particles")

    def __init__(self, rid, call, ret_am, est, particles):
        self.rid = rid
        self.call = call
        self.ret_am = ret_am
        self.future = cf.Future()
        self.est = est
        self.arrival = time.perf_counter()
        self.start = None
        self.end = None
        self.bypassed = 0
        self.particles = particles


def native_executor(device=0, pm_budget_bytes=2 << 30):
    """Executor factory: one native slot per worker, created on first use."""
    local = threading.local()
    made = []
    lock = threading.Lock()

    def run(call: FofCall, ret_am=False):
        """The fof_with_info result of one request (catalogue sorted on the
        device) and the slot's peak device memory."""
        if not hasattr(local, "slot"):
            local.slot = _native.slot_create(device, pm_budget_bytes)
            with lock:
                made.append(local.slot)
        try:
            out = _catalogue_call(call, ret_am, slot=local.slot)
        finally:
            peak = _native.slot_stat(local.slot, "peak_bytes")
        return out, peak

    run.returns_result = True

    def close():
        with lock:
            for s in made:
                _native.slot_destroy(s)
            made.clear()

    run.close = close
    return run


class Server:
    """Continuous-batching server of `fof_with_info` requests.

    slots:       concurrent requests on the GPU
    hbm_budget:  device bytes the running requests may hold together
                 (default: 80 % of the free device memory at start)
    executor:    callable(FofCall) -> ((in_halo, halo_id, ang_mom, ierr),
                 peak_bytes); the native slots by default (those return the
                 finished result, its catalogue sorted on the device)
    """

    FOF_BYTES = 200.0    # initial per-particle estimates (device bytes)
    BOUND_BYTES = 450.0

    def __init__(self, slots=4, hbm_budget=None, device=0, pm_budget_bytes=2 << 30, executor=None,
                 max_bypass=8):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.slots = slots
        self.max_bypass = max_bypass
        self.pm_budget = pm_budget_bytes if executor is None else 0
        if hbm_budget is None:
            if executor is None:
                import torch
                free, _ = torch.cuda.mem_get_info(device)
                hbm_budget = int(0.8 * free)
            else:
                hbm_budget = 1 << 40
        self.budget = int(hbm_budget)
        self._exec = executor or native_executor(device, pm_budget_bytes)
        self._per_particle = {False: self.FOF_BYTES, True: self.BOUND_BYTES}
        self._cv = threading.Condition()
        self._queue = collections.deque()
        self._reserved = 0
        self._running = 0
        self._closed = False
        self._next_id = 0
        self.done = []           # finished requests, in completion order
        self.max_running = 0
        self.max_reserved = 0
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(slots)]
        for w in self._workers:
            w.start()

    # ---------------------------------------------------------------- API
    def submit(self, xp_list, **kw) -> cf.Future:
        """Queue one `fof_with_info(xp_list, **kw)` request; the future
        yields its result dict (or raises its error)."""
        ret_am = bool(kw.get("return_ang_mom", False))
        try:
            call = _prepare(xp_list, check_masses=False, device_units=True, **kw)
        except (ValueError, TypeError) as exc:
            f = cf.Future()
            f.set_exception(exc)
            return f
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            rid = self._next_id
            self._next_id += 1
            if not isinstance(call, FofCall):  # total_np == 0: the final result already
                f = cf.Future()
                f.set_result(catalogue_from_ids(*call, return_ang_mom=ret_am))
                return f
            n = int(call.total_np)
            req = _Request(rid, call, ret_am, self._estimate(n, bool(call.bound_check)), n)
            self._queue.append(req)
            self._cv.notify_all()
        return req.future

    def close(self, wait=True):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for w in self._workers:
                w.join()
        close = getattr(self._exec, "close", None)
        if close:
            close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def latencies_ms(self):
        """(arrival -> done) latency of every finished request, ms."""
        return [1e3 * (r.end - r.arrival) for r in self.done]

    # ----------------------------------------------------------- internals
    def _estimate(self, n, bound):
        est = self._per_particle[bound] * n + (64 << 20)
        if bound:
            est += self.pm_budget
        return int(est)

    def _pick(self):
        """Next admissible request (lock held), or None."""
        if not self._queue:
            return None
        free = self.budget - self._reserved
        head = self._queue[0]
        if head.est > self.budget:  # runs alone
            return head if self._running == 0 else None
        if head.est <= free:
            return head
        if head.bypassed >= self.max_bypass:
            return None
        for r in list(self._queue)[1:]:
            if r.est <= free:
                head.bypassed += 1
                return r
        return None

    def _work(self):
        while True:
            with self._cv:
                while True:
                    if self._closed and not self._queue:
                        return
                    req = self._pick()
                    if req is not None:
                        break
                    self._cv.wait()
                self._queue.remove(req)
                self._reserved += req.est
                self._running += 1
                self.max_running = max(self.max_running, self._running)
                self.max_reserved = max(self.max_reserved, self._reserved)
                req.start = time.perf_counter()
            peak = 0
            try:
                if getattr(self._exec, "returns_result", False):
                    out, peak = self._exec(req.call, req.ret_am)
                else:
                    (ih, hid, am, ierr), peak = self._exec(req.call)
                    res = _finish(req.call, ih, hid, am, ierr)
                    out = catalogue_from_ids(*res, return_ang_mom=req.ret_am)
                err = None
            except Exception as exc:  # delivered through the future
                out, err = None, exc
            req.end = time.perf_counter()
            with self._cv:
                self._reserved -= req.est
                self._running -= 1
                if peak and req.particles:
                    b = bool(req.call.bound_check)
                    extra = self.pm_budget if b else 0
                    per = max(0.0, (peak - extra) / req.particles)
                    self._per_particle[b] = max(self._per_particle[b], per)
                self.done.append(req)
                self._cv.notify_all()
            if err is None:
                req.future.set_result(out)
            else:
                req.future.set_exception(err)


def percentile(values, q):
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if len(values) else float("nan")
