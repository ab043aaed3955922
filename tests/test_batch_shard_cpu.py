"""Sharding the batch over ranks (host logic, no GPU): the assignment is
deterministic and balanced, and the results of a world-size-2 run over the
gloo backend come back complete, in instance order, equal to a 1-rank run.
The per-shard solve is replaced by the oracle's CG (the batched GPU solver
is tested in test_gpu_batch.py)."""
import os
import socket

import numpy as np
import pytest

import oracle as O


def _instances(nb=9, seed=11):
    rng = np.random.default_rng(seed)
    ns = rng.integers(3, 14, size=nb)
    meshes = [O.unit_square(int(n), int(n)) for n in ns]
    kappas = [np.exp(rng.standard_normal(m.cells.shape[0])) for m in meshes]
    fs = [rng.uniform(-1, 1, m.coords.shape[0]) for m in meshes]
    return meshes, kappas, fs


class _Res:
    def __init__(self, sols, its, rels):
        self.solutions, self.iterations, self.rel_residuals = sols, its, rels
        self.statuses = np.zeros(len(sols), np.int32)


def _oracle_solve(ms, ks, fs):
    sols, its, rels = [], [], []
    for m, k, f in zip(ms, ks, fs):
        A = O.assemble_stiffness_2d(m, k)
        b = O.assemble_rhs_2d_values(m, np.repeat(f[m.cells].mean(axis=1, keepdims=True), 3, axis=1))
        bd = O.boundary_dofs_2d(m)
        Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
        x, it, res = O.solve_cg(Ab, bb, None, 1e-10, 10000)
        sols.append(x)
        its.append(it)
        rels.append(res / max(np.linalg.norm(bb), 1e-300))
    return _Res(sols, np.array(its), np.array(rels))


def test_shard_assignment_is_balanced_and_deterministic(fcu):
    costs = np.array([9, 1, 7, 7, 3, 2, 8, 5, 4], float)
    a = fcu.shard_instances(costs, 3)
    assert a == fcu.shard_instances(costs, 3)
    assert sorted(i for sh in a for i in sh) == list(range(len(costs)))
    loads = [costs[sh].sum() for sh in a]
    assert max(loads) - min(loads) <= costs.max()
    assert fcu.shard_instances(costs, 1) == [list(range(len(costs)))]
    assert fcu.shard_instances([], 2) == [[], []]
    with pytest.raises(ValueError):
        fcu.shard_instances(costs, 0)


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "fenics-rs_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    import fenics_cuda as fcu
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        meshes, kappas, fs = _instances()
        sols, its, rels, sts = fcu.solve_poisson_batch_sharded(meshes, kappas, fs, rank=rank, world=world,
                                                              solve=_oracle_solve)
        q.put((rank, [s.tolist() for s in sols], its.tolist(), sts.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_two_ranks_gloo(fcu):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    meshes, kappas, fs = _instances()
    sols1, its1, _, _ = fcu.solve_poisson_batch_sharded(meshes, kappas, fs, solve=_oracle_solve)
    for rank, sols, its, sts in out:
        assert len(sols) == len(meshes) and sts == [0] * len(meshes)
        assert its == its1.tolist()
        for a, b in zip(sols, sols1):
            assert np.array_equal(np.asarray(a), b)
