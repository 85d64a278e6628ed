"""Sharding of a dataset over ranks (world size 2, gloo on CPU): every structure is solved
by exactly one rank, the packing balances voxels, and the gathered results are in input
order on every rank. The per-rank solve is a stand-in that needs no GPU; the GPU solve
itself is covered by tests/test_gpu_batched.py."""

import os
import socket

import numpy as np
import pytest


def fake_solve(lms, mus, grids, **kwargs):
    """Deterministic per-structure outputs: C = (mean lambda + 2 mean mu) * I, iters = nx."""
    c = np.stack([np.eye(6) * (float(np.mean(l)) + 2.0 * float(np.mean(m)))
                  for l, m in zip(lms, mus)])
    it = np.array([[g.nx] * 6 for g in grids], dtype=np.int32)
    st = np.ones((len(lms), 6), dtype=np.int32)
    return c, it, st


def dataset(n=11, seed=0):
    from jaxmaterials_b200 import GridSpec

    rng = np.random.default_rng(seed)
    sizes = rng.choice([4, 6, 8, 12], size=n)
    lms = [np.full((s, s, s), float(i), np.float32) for i, s in enumerate(sizes)]
    mus = [np.full((s, s, s), 0.5 * i, np.float32) for i, s in enumerate(sizes)]
    grids = [GridSpec(int(s), int(s), int(s), float(s), float(s), float(s)) for s in sizes]
    return lms, mus, grids


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from jaxmaterials_b200.solver.distributed import c_eff_batch_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lms, mus, grids = dataset()
        C, it, st, owner = c_eff_batch_sharded(lms, mus, grids, solve=fake_solve)
        q.put((rank, C, it, st, owner))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_lpt_balances():
    from jaxmaterials_b200.solver.distributed import assign_lpt

    work = [128 ** 3] * 3 + [64 ** 3] * 10 + [32 ** 3] * 20
    owner = assign_lpt(work, 4)
    loads = np.bincount(owner, weights=work, minlength=4)
    assert loads.max() - loads.min() <= 128 ** 3
    assert set(owner) == {0, 1, 2, 3}
    assert (assign_lpt(work, 1) == 0).all()


@pytest.mark.timeout(120)
def test_sharded_dataset_world2():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    lms, mus, grids = dataset()
    C_ref, it_ref, st_ref = fake_solve(lms, mus, grids)
    owners = []
    for rank, C, it, st, owner in res:
        np.testing.assert_array_equal(C, C_ref)
        np.testing.assert_array_equal(it, it_ref)
        np.testing.assert_array_equal(st, st_ref)
        owners.append(owner)
    np.testing.assert_array_equal(owners[0], owners[1])
    assert set(owners[0]) == {0, 1}
