"""The multi-GPU sweep path end to end: two ranks of a gloo process group, both on
cuda:0 (one GPU per call here), each tracing its cost-balanced shard of one sweep's
angles with the real kernels, the fields gathered to rank 0.  The merged sweep must
equal one sbr_run of the whole job bit for bit: every sample's field is an integer
fixed-point sum that does not depend on which rank or launch traced it.  Replaces
the reference's MPI partition and gather (src/app/sweep.cu:172-179, :465-547).
The two ranks' kernels are independent sweeps; neither waits on the other."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _job():
    from sagittasbr_b200 import meshes as M
    import sagittasbr_b200 as sbr
    v, t = M.trihedral(1.0, 20)
    th, ph = np.meshgrid(np.linspace(0.0, 90.0, 7), np.linspace(0.0, 90.0, 6), indexing="ij")
    return v, t, sbr.JobSpec(th.ravel(), ph.ravel(), [8e9, 1e10, 1.2e10], 160, 160, 2.0 * M.bounding_radius(v), 3)


def _worker(rank, world, port, balance, q):
    import datetime

    import torch
    import torch.distributed as dist

    import sagittasbr_b200 as sbr
    from sagittasbr_b200 import sharding as S
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        v, t, job = _job()
        with sbr.Scene(v, t, device=0) as sc:
            merged = S.sharded_sweep(sc, job, rank, world, balance=balance)
            sp = S.ShardedPlan(sc, job, rank, world, balance=balance)
            sp.execute()
            dev = sp.gather(torch)
            sp.execute()  # a plan runs again without reset
            dev2 = sp.gather(torch)
            parts = sp.parts
            sp.close()
            if rank == 0:
                whole = sbr.run(sc, job).field.reshape(len(job.theta_deg), len(job.freqs_hz))
                q.put((merged, dev, dev2, whole, parts))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("balance", ["block", "cost"])
def test_two_ranks_on_one_gpu_equal_one_run(balance):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, balance, q)) for r in range(world)]
    for p in procs:
        p.start()
    merged, dev, dev2, whole, parts = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(c > 0 for _, c in parts) and sum(c for _, c in parts) == whole.shape[0]
    np.testing.assert_array_equal(merged, whole)
    np.testing.assert_array_equal(dev, whole)
    np.testing.assert_array_equal(dev2, whole)
