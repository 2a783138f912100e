"""
Multi-process sharding on CPU: two gloo ranks split a population and an
image exactly as GPU ranks would, evaluating with the reference DLL oracle
instead of the GPU engine, and must reproduce the single-process results.
"""

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_population(model, subset):
    from helpers import load_info, marshal, normalise, reference_raw
    info = load_info(model)
    out = []
    for q, pars in subset:
        raw = reference_raw(model, info, [q], pars)
        _, values, _ = marshal(info, pars, [q])
        out.append(normalise(raw, 2, len(q), values)["I"])
    return out


def _worker(rank, size, port, queue):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        from helpers import load_info, marshal, reference_raw
        import numpy as np
        from sasmodels_b200 import multigpu, workloads
        pop = [(q, p) for name, q, p in workloads.population(n_sets=10, seed=2, max_pd_n=4)
               if name == "ellipsoid"]
        pop = [(q[::9], p) for q, p in pop]
        curves = multigpu.evaluate_population("ellipsoid", pop, evaluate=_oracle_population)
        name, qv, pars = workloads.cylinder_2d(n=6, radius_n=3, length_n=3, theta_n=3, phi_n=3)
        info = load_info(name)
        raw = multigpu.evaluate_image(
            qv, lambda qb: reference_raw(name, info, qb, pars))
        # one call's mesh split over the ranks, partial sums from the
        # reference DLL's own restart contract (pd_start > 0 accumulates)
        from oracle import refdll
        name1, (q1,), pars1 = workloads.sphere_1d()
        info1 = load_info(name1)
        d1, v1, _ = marshal(info1, pars1, [q1])
        dll = refdll.load(name1)
        mesh = multigpu.evaluate_mesh(
            d1.num_eval, lambda lo, hi: dll.call("Iq", q1, d1.buffer, v1, 2, pd_start=lo,
                                                 pd_stop=hi, result=np.zeros(2*len(q1) + 4)))
        # a 1D image returning <F> and <F^2> (nout = 2) with fewer q points
        # than ranks: rank 1's block is empty
        tiny = multigpu.evaluate_image(
            [q1[:1]], lambda qb: reference_raw(name1, info1, qb, pars1), nout=2)
        queue.put((rank, [c.tolist() for c in curves], raw.tolist(), mesh.tolist(),
                   tiny.tolist()))
    finally:
        dist.destroy_process_group()


def test_shard_by_cost_balances():
    from sasmodels_b200.multigpu import shard_by_cost
    costs = [10, 9, 1, 1, 1, 8, 2]
    parts = shard_by_cost(costs, 2)
    assert sorted(sum(parts, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 2
    assert shard_by_cost(costs, 2) == parts      # deterministic


def test_two_rank_gloo_matches_single_process():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import load_info, reference_raw
    from sasmodels_b200 import multigpu, workloads
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # single-process reference
    pop = [(q, p) for name, q, p in workloads.population(n_sets=10, seed=2, max_pd_n=4)
           if name == "ellipsoid"]
    pop = [(q[::9], p) for q, p in pop]
    single = _oracle_population("ellipsoid", pop)
    name, qv, pars = workloads.cylinder_2d(n=6, radius_n=3, length_n=3, theta_n=3, phi_n=3)
    raw_single = reference_raw(name, load_info(name), qv, pars)
    name1, (q1,), pars1 = workloads.sphere_1d()
    mesh_single = reference_raw(name1, load_info(name1), [q1], pars1)
    tiny_single = reference_raw(name1, load_info(name1), [q1[:1]], pars1)
    meshes = []
    for rank, curves, raw, mesh, tiny in results:
        np.testing.assert_array_equal(np.array(tiny), tiny_single)
        assert len(curves) == len(single)
        for a, b in zip(curves, single):
            np.testing.assert_array_equal(np.array(a), b)
        np.testing.assert_array_equal(np.array(raw), raw_single)
        # the two partial sums re-associate the mesh sum: equal to rounding
        np.testing.assert_allclose(np.array(mesh), mesh_single, rtol=1e-13, atol=0)
        meshes.append(mesh)
    assert meshes[0] == meshes[1]        # identical on every rank


def test_mesh_ranges_cover():
    from sasmodels_b200.multigpu import mesh_ranges
    for n, r in [(35, 2), (490000, 8), (1, 4), (0, 3)]:
        rg = mesh_ranges(n, r)
        assert rg[0][0] == 0 and rg[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(rg[:-1], rg[1:]))


def _dp_worker(rank, size, port, queue):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        from sasmodels_b200 import multigpu
        # one flat bucket of several shapes (the loss, matrices, vectors)
        gen = torch.Generator().manual_seed(rank)
        grads = [torch.full((1,), float(rank + 1)), torch.arange(6.0).reshape(2, 3)*(rank + 1),
                 torch.randn(5, generator=gen)]
        multigpu.allreduce_mean(grads)

        class Net:
            synced = False

            def _sync_bf16(self):
                self.synced = True
        net = Net()
        net.params = [torch.randn(3, 4, generator=torch.Generator().manual_seed(10 + rank))]
        multigpu.broadcast_parameters(net)
        # data-parallel gradient descent of a least-squares model: each rank
        # takes its slice of every global batch, gradients averaged per step
        data = torch.Generator().manual_seed(99)
        X = torch.randn(64, 3, generator=data, dtype=torch.float64)
        y = torch.randn(64, generator=data, dtype=torch.float64)
        w = torch.zeros(3, dtype=torch.float64)
        for step in range(4):
            lo, hi = multigpu.batch_slice(step*16, 16, rank, size)
            r = X[lo:hi] @ w - y[lo:hi]
            g = 2.0*X[lo:hi].T @ r/(hi - lo)
            multigpu.allreduce_mean([g])
            w -= 0.1*g
        queue.put((rank, [t.tolist() for t in grads], net.params[0].tolist(), net.synced,
                   w.tolist()))
    finally:
        dist.destroy_process_group()


def test_data_parallel_helpers_two_ranks():
    import torch
    from sasmodels_b200.multigpu import batch_slice
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [[1.5], (torch.arange(6.0).reshape(2, 3)*1.5).tolist(),
              ((torch.randn(5, generator=torch.Generator().manual_seed(0))
                + torch.randn(5, generator=torch.Generator().manual_seed(1)))/2).tolist()]
    data = torch.Generator().manual_seed(99)
    X = torch.randn(64, 3, generator=data, dtype=torch.float64)
    y = torch.randn(64, generator=data, dtype=torch.float64)
    w = torch.zeros(3, dtype=torch.float64)
    for step in range(4):
        Xb, yb = X[step*16:(step + 1)*16], y[step*16:(step + 1)*16]
        w -= 0.1*(2.0*Xb.T @ (Xb @ w - yb)/16)
    params0 = torch.randn(3, 4, generator=torch.Generator().manual_seed(10)).tolist()
    for rank, grads, params, synced, w_dp in results:
        for a, b in zip(grads, expect):
            np.testing.assert_allclose(np.array(a), np.array(b), rtol=1e-6)
        assert params == params0 and synced
        np.testing.assert_allclose(w_dp, w.numpy(), rtol=1e-12, atol=1e-15)
    # every rank holds the same bits after the reduction
    assert results[0][1] == results[1][1] and results[0][4] == results[1][4]
    # the slices of a global batch are equal and cover it
    assert [batch_slice(32, 16, r, 4) for r in range(4)] == [(32, 36), (36, 40), (40, 44),
                                                            (44, 48)]
    with pytest.raises(ValueError):
        batch_slice(0, 10, 0, 4)
