"""Serving loop on the GPU: requests of mixed sizes, FoF-only and with
unbinding, cube and physical units, run concurrently on native slots; each
result equals the same request run alone through fof_with_info (FoF exactly;
unbinding within the particle-mesh tolerance: the deposit's atomic order may
flip a marginally bound member)."""
import numpy as np
import pytest

import py_fof_b200 as P
from py_fof_b200 import serve, workloads as W

pytestmark = pytest.mark.gpu


def _requests():
    rng = np.random.default_rng(11)
    reqs = []
    for k in range(14):
        n = int(10 ** rng.uniform(3.5, 5.3))
        L = float(round(n ** (1 / 3), 3))
        bound = k % 2 == 1
        d = W.plummer_box(n, L, max(1, n // 4096), seed=500 + k, with_velocities=bound,
                          lognormal_mass=0.3 if bound else None)
        kw = dict(L_Box=L, linking_length=0.2, np_halo_min=10, return_ang_mom=True)
        if bound:
            kw.update(vp_list=d["vp"], mp_list=d["mp"], bound_check=True, ng_global=512.0)
            if k % 4 == 3:
                kw.update(units="physical", softening=0.05, L_Box=L * 1.5)
        reqs.append((d["xp"], kw))
    # a list input with a particle-mesh halo
    xs, vs = W.nfw_halos(5, seed=3, sizes=[40, 2500, 300, 1200, 90])
    reqs.append((xs, dict(vp_list=vs, L_Box=512.0, bound_check=True, return_ang_mom=True)))
    return reqs


def _close(a, b, bound):
    if not bound:
        assert a["nhalo_found"] == b["nhalo_found"]
        assert np.array_equal(a["in_halo"], b["in_halo"])
        assert all(np.array_equal(x, y) for x, y in zip(a["halo_indices"], b["halo_indices"]))
        assert np.allclose(a["ang_mom"], b["ang_mom"], rtol=1e-9, atol=1e-12)
    else:
        n_in = int(b["in_halo"].sum())
        assert int((a["in_halo"] != b["in_halo"]).sum()) <= max(2, n_in // 1000)
        assert abs(a["nhalo_found"] - b["nhalo_found"]) <= 1


def test_served_equals_alone():
    reqs = _requests()
    alone = [P.fof_with_info(x, **kw) for x, kw in reqs]
    with serve.Server(slots=4) as s:
        futs = [s.submit(x, **kw) for x, kw in reqs]
        served = [f.result(timeout=300) for f in futs]
        again = [s.submit(x, **kw).result(timeout=300) for x, kw in reqs[:3]]
    assert s.max_running >= 2
    for (x, kw), a, b in zip(reqs, served, alone):
        _close(a, b, kw.get("bound_check", False))
    for (x, kw), a, b in zip(reqs, again, alone):
        _close(a, b, kw.get("bound_check", False))
