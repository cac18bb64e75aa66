"""Serving loop on the GPU: requests of mixed sizes, FoF-only and with
unbinding, cube and physical units, run concurrently on native slots; each
result equals the same request run alone through fof_with_info, bit for bit
(membership, halo ids and catalogue; the particle-mesh deposit adds
fixed-point integers, so no result depends on how work interleaves on the
device).  A sample of the requests is also checked against the oracle."""
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


def _same(a, b):
    assert a["nhalo_found"] == b["nhalo_found"]
    assert np.array_equal(a["in_halo"], b["in_halo"])
    assert all(np.array_equal(x, y) for x, y in zip(a["halo_indices"], b["halo_indices"]))
    assert np.allclose(a["ang_mom"], b["ang_mom"], rtol=1e-9, atol=1e-12)


def test_served_equals_alone():
    reqs = _requests()
    alone = [P.fof_with_info(x, **kw) for x, kw in reqs]
    with serve.Server(slots=4) as s:
        futs = [s.submit(x, **kw) for x, kw in reqs]
        served = [f.result(timeout=300) for f in futs]
        again = [s.submit(x, **kw).result(timeout=300) for x, kw in reqs[:3]]
    assert s.max_running >= 2
    for a, b in zip(served, alone):
        _same(a, b)
    for a, b in zip(again, alone):
        _same(a, b)


def test_served_against_oracle():
    """Served results of FoF-only and unbinding requests against the oracle:
    FoF bit-exact; unbinding bit-exact for direct-summation candidates (the
    library's default FP64 path) and within the energy band elsewhere."""
    from tests.helpers import check_unbinding_band, oracle_core_diag
    reqs = _requests()
    pick = [0, 1, 2, 3, 5, 7, len(reqs) - 1]
    with serve.Server(slots=4) as s:
        futs = [s.submit(reqs[i][0], **reqs[i][1]) for i in pick]
        served = [f.result(timeout=300) for f in futs]
    for i, r in zip(pick, served):
        x, kw = reqs[i]
        o, energy, scale = oracle_core_diag(x, **kw)
        g = (r["in_halo"], np.zeros_like(o[1]))
        for hid, idx in enumerate(r["halo_indices"], start=1):
            g[1][idx] = hid
        if kw.get("bound_check", False):
            check_unbinding_band(g, o, energy, scale)
        else:
            assert np.array_equal(g[1], o[1])
