"""Multi-GPU host logic on CPU: two gloo ranks (127.0.0.1).

Each rank takes its shard of the 64-member ensemble and of a request list,
advances its members with the oracle (tiny grids), and the whole-job rate is
the sum of the ranks' work over the max of their times.  Checks: the shards
cover every member exactly once, the reductions are the max and the sum, and a
member's result does not depend on which rank ran it.
"""

import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, outdir):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    sys.path[:0] = [os.path.join(repo, "oracle"), os.path.join(repo, "boundarylayerdynamics.jl_b200")]
    import bld_oracle as O
    from BoundaryLayerDynamics import replicas, workloads
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    groups = workloads.ensemble_members()
    mine = replicas.shard_groups(groups, world, rank)
    ids = []
    for gi, g in enumerate(groups):
        lo, hi = replicas.shard(len(g["z0"]), world, rank)
        ids += [(gi, i) for i in range(lo, hi)]
    # advance two of this rank's members of the smallest class on a tiny grid with the oracle
    results = {}
    spec0 = workloads.les_spec(8, 4, (2 * np.pi, np.pi, 1.0))
    for gi, i in ids[:2]:
        z0, cs = float(groups[gi]["z0"][i]), float(groups[gi]["cs"][i])
        spec = dict(spec0, lower=("rough", z0), sgs=dict(Cs=cs))
        m = workloads.build(spec, O)
        u, v, w = workloads.initial_fields(spec, seed=1000 * gi + i)
        m.initialize(vel1=u, vel2=v, vel3=w)
        m.evolve(3 * 1e-3, 1e-3)
        results[f"{gi}_{i}"] = m.state["vel1"]
    t = 0.5 + rank                 # a stand-in for the rank's timed region
    rate = replicas.whole_job_rate(100.0 * (rank + 1), t, dist)
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), ids=np.array(ids), rate=rate,
             tmax=replicas.reduce_max(t, dist), nmine=sum(len(g["z0"]) for g in mine), **results)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_balanced():
    from BoundaryLayerDynamics import replicas
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    r = [np.load(tmp_path / f"rank{k}.npz") for k in range(world)]
    ids = [tuple(x) for k in range(world) for x in r[k]["ids"]]
    assert len(ids) == 64 and len(set(ids)) == 64                 # every member exactly once
    assert r[0]["nmine"] + r[1]["nmine"] == 64
    for k in range(world):
        assert float(r[k]["tmax"]) == 1.5                          # max over ranks
        assert float(r[k]["rate"]) == pytest.approx(300.0 / 1.5)   # sum of work / slowest rank
    # the same member run by a single process gives the same result
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import bld_oracle as O
    from BoundaryLayerDynamics import workloads
    groups = workloads.ensemble_members()
    key = [k for k in r[1].files if "_" in k and k[0].isdigit()][0]
    gi, i = map(int, key.split("_"))
    spec = dict(workloads.les_spec(8, 4, (2 * np.pi, np.pi, 1.0)), lower=("rough", float(groups[gi]["z0"][i])),
                sgs=dict(Cs=float(groups[gi]["cs"][i])))
    m = workloads.build(spec, O)
    u, v, w = workloads.initial_fields(spec, seed=1000 * gi + i)
    m.initialize(vel1=u, vel2=v, vel3=w)
    m.evolve(3 * 1e-3, 1e-3)
    assert np.array_equal(m.state["vel1"], r[1][key])
