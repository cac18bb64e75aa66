"""Serving loop (py_fof_b200.serve) on CPU: the scheduler, admission by the
memory budget and the result path, with the CPU oracle as the executor."""
import threading
import time

import numpy as np
import pytest

from oracle import oracle as O
from py_fof_b200 import serve, workloads as W
from tests.helpers import oracle_fof_with_info


class OracleExec:
    """Executor computing a FofCall with the oracle; optional delay to make
    requests overlap; records how many run at once."""

    def __init__(self, delay=0.0, peak=0):
        self.delay = delay
        self.peak = peak
        self.lock = threading.Lock()
        self.now = 0
        self.most = 0

    def __call__(self, call):
        with self.lock:
            self.now += 1
            self.most = max(self.most, self.now)
        try:
            time.sleep(self.delay)
            if call.mp is not None and not np.all(np.isfinite(call.mp) & (call.mp > 0)):
                n = call.total_np
                return (np.zeros(n, np.int32), np.zeros(n, np.int32),
                        np.zeros((3, call.nhalo)), 5), self.peak
            call = call.on_host()
            vp, mp = call.dense()
            out = O.fof_fortran(np.asfortranarray(call.xp), np.asfortranarray(vp), mp, call.np_halo,
                                call.nhalo, call.L_Box, call.link, call.np_halo_min, call.bound_check,
                                call.verbose, call.softening, call.a_val, call.b_val, call.s_15_val,
                                call.n_threads, call.total_np, call.ng_val, call.ng_global_val)
            return tuple(out), self.peak
        finally:
            with self.lock:
                self.now -= 1


def _requests(seed=0, count=10):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        n = int(10 ** rng.uniform(3, 4.2))
        L = float(round(n ** (1 / 3), 3))
        halos = max(1, n // 4096)
        bound = k % 2 == 1
        d = W.plummer_box(n, L, halos, seed=seed * 100 + k, with_velocities=bound,
                          lognormal_mass=0.3 if bound else None)
        kw = dict(L_Box=L, linking_length=0.2, np_halo_min=10, return_ang_mom=True)
        if bound:
            kw.update(vp_list=d["vp"], mp_list=d["mp"], bound_check=True, ng_global=512.0)
            if k % 4 == 3:
                kw.update(units="physical", softening=0.05, L_Box=L * 1.5)
        reqs.append((d["xp"], kw))
    return reqs


def _same(a, b):
    assert a["nhalo_found"] == b["nhalo_found"]
    assert np.array_equal(a["in_halo"], b["in_halo"])
    assert np.array_equal(a["np_per_halo"], b["np_per_halo"])
    assert all(np.array_equal(x, y) for x, y in zip(a["halo_indices"], b["halo_indices"]))
    assert np.allclose(a["ang_mom"], b["ang_mom"], rtol=1e-12, atol=0)


def test_results_alone_and_in_the_mix():
    reqs = _requests(1)
    ex = OracleExec(delay=0.02)
    with serve.Server(slots=3, executor=ex) as s:
        futs = [s.submit(x, **kw) for x, kw in reqs]
        res = [f.result(timeout=120) for f in futs]
    for (x, kw), r in zip(reqs, res):
        _same(r, oracle_fof_with_info(x, **kw))
    assert ex.most >= 2  # requests overlapped
    assert len(s.done) == len(reqs)


def test_budget_limits_concurrency():
    reqs = _requests(2, count=8)
    ex = OracleExec(delay=0.03)
    sizes = [x.shape[1] for x, _ in reqs]
    budget = int(serve.Server.BOUND_BYTES * max(sizes) * 2.5) + (64 << 21)
    with serve.Server(slots=6, hbm_budget=budget, executor=ex) as s:
        for f in [s.submit(x, **kw) for x, kw in reqs]:
            f.result(timeout=120)
    assert s.max_reserved <= budget
    assert s.max_running <= 6


def test_bypass_is_bounded():
    """A large head request is passed by at most max_bypass later ones."""
    ex = OracleExec(delay=0.05)
    rng = np.random.default_rng(5)
    small = [rng.uniform(0, 5, (3, 300)) for _ in range(6)]
    big = rng.uniform(0, 30, (3, 20000))
    est_small = serve.Server.FOF_BYTES * 300 + (64 << 20)
    est_big = serve.Server.FOF_BYTES * 20000 + (64 << 20)
    budget = int(est_big + est_small) - 1  # the big one cannot run beside a small one
    with serve.Server(slots=2, hbm_budget=budget, executor=ex, max_bypass=2) as s:
        f0 = s.submit(small[0], L_Box=5.0)
        time.sleep(0.01)  # small[0] is running when the big one arrives
        fb = s.submit(big, L_Box=30.0)
        fs = [s.submit(x, L_Box=5.0) for x in small[1:]]
        for f in [f0, fb] + fs:
            f.result(timeout=120)
    order = [r.rid for r in s.done]
    # the big request (id 1) finished after at most 2 + 1 small ones
    assert order.index(1) <= 3


def test_oversized_request_runs_alone():
    reqs = _requests(3, count=6)
    ex = OracleExec(delay=0.02)
    with serve.Server(slots=4, hbm_budget=1 << 20, executor=ex, max_bypass=2) as s:
        futs = [s.submit(x, **kw) for x, kw in reqs]
        for f in futs:
            f.result(timeout=120)
    # every request exceeds the budget: each ran with nothing beside it
    assert len(s.done) == len(reqs)
    assert s.max_running == 1 and ex.most == 1


def test_errors_stay_with_their_request():
    reqs = _requests(4, count=4)
    x, kw = reqs[1]
    bad = dict(kw)
    mp = np.array(kw["mp_list"], copy=True)
    mp[3] = -1.0
    bad["mp_list"] = mp
    with serve.Server(slots=2, executor=OracleExec()) as s:
        f_bad = s.submit(x, **bad)
        f_inv = s.submit(np.zeros((2, 5)), L_Box=10.0)
        f_ok = [s.submit(x2, **kw2) for x2, kw2 in reqs]
        with pytest.raises(ValueError, match="positive and finite"):
            f_bad.result(timeout=60)
        with pytest.raises(ValueError):
            f_inv.result(timeout=60)
        for (x2, kw2), f in zip(reqs, f_ok):
            _same(f.result(timeout=60), oracle_fof_with_info(x2, **kw2))


def test_empty_request():
    with serve.Server(slots=1, executor=OracleExec()) as s:
        r = s.submit(np.zeros((3, 0))).result(timeout=10)
    assert r["nhalo_found"] == 0
