"""List inputs split across ranks (world size 2 and 3, gloo on CPU): the
partition, the halo-id shift and the output exchange reproduce the single
call exactly.  The per-rank computation is the CPU oracle here (the GPU path
is exercised by test_shard_gpu.py); what is tested is the host logic of
py_fof_b200.shard."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from py_fof_b200 import shard, workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(kind):
    if kind == "fof":
        rng = np.random.default_rng(0)
        xs = []
        for k, n in enumerate([300, 5, 2000, 40, 0, 900, 12, 700]):
            # a few tight clumps plus scattered particles per region
            c = rng.uniform(0, 6, (3, 4))
            x = c[:, rng.integers(0, 4, n)] + rng.normal(0, 0.25, (3, n))
            x[:, ::5] = rng.uniform(0, 6, (3, len(x[0, ::5])))
            xs.append(x + 40.0 * k)
        return xs, dict(L_Box=512.0, linking_length=0.3, np_halo_min=10, return_ang_mom=True)
    xs, vs = W.nfw_halos(9, seed=4, sizes=[25, 300, 1200, 60, 15, 2500, 80, 400, 30])
    ms = [np.random.default_rng(k).lognormal(0, 0.3, x.shape[1]) for k, x in enumerate(xs)]
    return xs, dict(vp_list=vs, mp_list=ms, L_Box=512.0, linking_length=0.2, np_halo_min=10,
                    bound_check=True, return_ang_mom=True)


def _worker(rank, world, port, kind, out):
    import torch.distributed as dist
    from tests.helpers import oracle_core
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        xs, kw = _case(kind)
        ih, hid, am = shard.fof_core_sharded(xs, core=oracle_core, **kw)
        np.savez(f"{out}_{rank}.npz", ih=ih, hid=hid, am=am)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,world", [("fof", 2), ("fof", 3), ("bound", 2)])
def test_sharded_equals_single_call(tmp_path, kind, world):
    from tests.helpers import oracle_core
    out = str(tmp_path / "r")
    mp.start_processes(_worker, args=(world, _free_port(), kind, out), nprocs=world,
                       start_method="spawn", join=True)
    xs, kw = _case(kind)
    ih, hid, am = oracle_core(xs, **kw)
    for r in range(world):
        z = np.load(f"{out}_{r}.npz")
        assert np.array_equal(z["ih"], ih)
        assert np.array_equal(z["hid"], hid)
        assert np.array_equal(z["am"], am)
    assert hid.max() > 3


def test_partition_regions():
    p = shard.partition_regions([10, 10, 10, 10], 2)
    assert p == [(0, 2), (2, 4)]
    p = shard.partition_regions([1000, 1, 1, 1], 2)
    assert p[0] == (0, 1) and p[1] == (1, 4)
    p = shard.partition_regions([5, 5], 4)
    assert [e - s for s, e in p] == [0, 1, 0, 1] or sum(e - s for s, e in p) == 2
    assert p[0][0] == 0 and p[-1][1] == 2
    for a, b in zip(p, p[1:]):
        assert a[1] == b[0]
