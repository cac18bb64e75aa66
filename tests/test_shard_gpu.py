"""List input split across two ranks that both run the native library on
the one GPU of the test box (gloo for the output exchange; the ranks'
kernels never wait on each other): the result equals the single call bit
for bit in membership and halo ids (each halo's unbinding does not depend on
which halos share its batch: the particle-mesh deposit adds fixed-point
integers)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from py_fof_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    xs, vs = W.nfw_halos(12, seed=6, sizes=[25, 300, 1500, 60, 15, 2500, 80, 400, 30, 5000, 120, 45])
    return xs, dict(vp_list=vs, L_Box=512.0, linking_length=0.2, np_halo_min=10, bound_check=True,
                    return_ang_mom=True)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from py_fof_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        xs, kw = _case()
        ih, hid, am = shard.fof_core_sharded(xs, **kw)
        np.savez(f"{out}_{rank}.npz", ih=ih, hid=hid, am=am)
    finally:
        dist.destroy_process_group()


def test_sharded_native_equals_single_call(tmp_path):
    import py_fof_b200 as P
    out = str(tmp_path / "r")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    xs, kw = _case()
    ih, hid, am = P._fof_core(xs, **kw)
    assert hid.max() > 5
    for r in range(2):
        z = np.load(f"{out}_{r}.npz")
        assert np.array_equal(z["ih"], ih)
        assert np.array_equal(z["hid"], hid)
        assert np.allclose(z["am"], am, rtol=1e-9, atol=1e-9 * np.abs(am).max())
