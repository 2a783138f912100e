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
        queue.put((rank, [c.tolist() for c in curves], raw.tolist(), mesh.tolist()))
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
    meshes = []
    for rank, curves, raw, mesh in results:
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
