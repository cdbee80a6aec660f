"""Ensembles and served requests on the device.

* member slots: per-member parameters set after creation, the active mask,
  per-member preparation and per-member divergence;
* uneven ensembles stepped by one parent graph per step equal each class
  stepped on its own, and the FP64 oracle;
* served requests: each result is the same alone and in a mix of concurrent
  requests (bitwise in practice; the bar is 1e-12 relative for FP64 and 1e-6
  for the mixed form), and equal to the FP64 oracle within the trajectory bar.
"""

import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

DT = 1e-3
TRAJ_TOL = 1e-9


@pytest.fixture(scope="module")
def BLD():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as B
    return B


def _spec(n=16, n3=8, **kw):
    from BoundaryLayerDynamics import workloads
    return workloads.les_spec(n, n3, (2 * math.pi, math.pi, 1.0), **kw)


def _ic(spec, seed):
    from BoundaryLayerDynamics import workloads
    return workloads.initial_fields(spec, seed)


def _load(model, fields, member=0):
    for f, v in zip(("vel1", "vel2", "vel3"), fields):
        model.set_field(f, v, member=member)


def _close(a, b, tol):
    for f in a:
        e = rel_l2(a[f], b[f])
        assert e <= tol, (f, e)


def test_member_params_after_creation(BLD):
    """set_member_params on a created handle equals per-member arrays at creation."""
    from BoundaryLayerDynamics import workloads
    spec = _spec()
    cs, z0, forcing = [0.09, 0.15], [3e-5, 5e-4], [0.7, 1.4]
    a = workloads.build(spec, BLD, members=2, member_cs=cs, member_z0=z0, member_forcing=forcing)
    b = workloads.build(spec, BLD, members=2)
    for m in range(2):
        b.set_member_params(m, cs=cs[m], z0=z0[m], forcing=forcing[m])
        for mod in (a, b):
            _load(mod, _ic(spec, 10 + m), member=m)
    a.evolve(10 * DT, DT)
    b.evolve(10 * DT, DT)
    for m in range(2):
        _close(a.get_state(m), b.get_state(m), 0.0)


@pytest.mark.parametrize("proj", ["auto", "pipe", "tile"])
def test_active_mask_and_prepare_member(BLD, proj, monkeypatch):
    """Inactive members keep their state; active ones equal a model of their own.
    `pipe` and `tile` force the projections of stored stage values onto the
    persistent k_project_pipe (whose blocks walk the items of active members
    only) or onto k_project_tile, 8 columns per block."""
    from BoundaryLayerDynamics import workloads
    if proj != "auto":
        monkeypatch.setenv("BLD_PROJ_TILE", "8")
        monkeypatch.setenv("BLD_PROJ_PIPE", "1" if proj == "pipe" else "0")
    spec = _spec()
    ens = workloads.build(spec, BLD, members=3)
    if proj != "auto":
        assert ens.kernels()["projection_stored"].startswith("k_project_" + proj), ens.kernels()
    for m in range(3):
        _load(ens, _ic(spec, 20 + m), member=m)
    ens.prepare()
    frozen = ens.get_state(1)
    ens.set_active([1, 0, 1])
    ens.step(12, DT)
    _close(ens.get_state(1), frozen, 0.0)
    for m in (0, 2):
        single = workloads.build(spec, BLD)
        _load(single, _ic(spec, 20 + m))
        single.evolve(12 * DT, DT)
        _close(ens.get_state(m), single.state, 1e-14)
    # a new request in slot 1: load, prepare it alone, switch it on, keep stepping
    _load(ens, _ic(spec, 99), member=1)
    ens.set_member_params(1, z0=2e-4, forcing=1.3)
    ens.prepare_member(1)
    ens.set_active([0, 1, 0])
    before0 = ens.get_state(0)
    ens.step(7, DT)
    _close(ens.get_state(0), before0, 0.0)
    single = workloads.build(dict(spec, lower=("rough", 2e-4), forcing=1.3), BLD)
    _load(single, _ic(spec, 99))
    single.evolve(7 * DT, DT)
    _close(ens.get_state(1), single.state, 1e-14)


def test_divergence_is_reported_per_member(BLD):
    from BoundaryLayerDynamics import workloads
    spec = _spec()
    ens = workloads.build(spec, BLD, members=3)
    for m in range(3):
        _load(ens, _ic(spec, 30 + m), member=m)
    ens.prepare()
    st = ens.get_state(2)
    st["vel1"][3, 2, 1] = np.inf
    ens.set_state(st, member=2)
    with pytest.raises(BLD.DivergenceError):
        ens.prepare_member(2)
    assert ens.diverged_members() == [2]
    with pytest.raises(BLD.DivergenceError):
        ens.step(1, DT)
    assert ens.diverged_members() == [2]
    assert ens.diverged_members() == []
    ens.set_active([1, 1, 0])            # the diverged member's slot is switched off
    ens.step(3, DT)                      # the others go on without error


def test_uneven_ensemble_one_graph_per_step(oracle, BLD):
    """Two size classes advanced by bld_ensemble_step equal each class on its own and the oracle."""
    from BoundaryLayerDynamics import workloads
    from BoundaryLayerDynamics.ensemble import Ensemble
    groups = [dict(spec=_spec(16, 8), z0=np.array([1e-4, 1e-3]), cs=np.array([0.1, 0.14])),
              dict(spec=_spec(24, 12), z0=np.array([2e-5]), cs=np.array([0.12]))]
    for precision in ("fp64",):
        ens = Ensemble.from_groups(groups, precision=precision)
        ens.initialize(groups, seed=40)
        ens.prepare()
        ens.step(15, DT)
        k = 0
        for g, model in zip(groups, ens.models):
            for i in range(model.members):
                s = dict(g["spec"], lower=("rough", float(g["z0"][i])), sgs=dict(Cs=float(g["cs"][i])))
                single = workloads.build(s, BLD, precision=precision)
                _load(single, _ic(s, 40 + k))
                single.evolve(15 * DT, DT)
                _close(model.get_state(i), single.state, 1e-14)
                if k == 2:
                    om = workloads.build(s, oracle)
                    u, v, w = _ic(s, 40 + k)
                    om.initialize(vel1=u, vel2=v, vel3=w)
                    om.evolve(15 * DT, DT)
                    _close(model.get_state(i), om.state, TRAJ_TOL)
                k += 1


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_served_request_same_alone_and_in_mix(oracle, BLD, precision, tol):
    """A request served alone and among concurrent requests gives the same result."""
    from BoundaryLayerDynamics import serving as S
    from BoundaryLayerDynamics import workloads
    sizes = ((16, 8), (24, 12))
    caps = {(16, 8): 3, (24, 12): 2}

    def server():
        pools = {s: workloads.build(S.spec_for(s), BLD, precision=precision, members=caps[s]) for s in sizes}
        return S.Server(pools, {s: 1 for s in sizes}, budget=10**12, dt=DT, tick=5, keep_results=True)

    def requests():
        return S.make_requests(12, rate=2000.0, seed=11, sizes=sizes, probs=(0.5, 0.5), steps=20)

    mix = requests()
    st = server().run(mix)
    assert st["completed"] == 12
    target = mix[7]
    # the target shared its pool with other requests for part of its run
    peers = [r for r in mix if r is not target and r.size == target.size
             and r.admitted < target.done and target.admitted < r.done]
    assert peers
    alone = [r for r in requests() if r.rid == target.rid]
    alone[0].arrival = 0.0
    assert server().run(alone)["completed"] == 1
    _close(target.result, alone[0].result, tol)
    if precision == "fp64":
        s = S.spec_for(target.size, z0=target.z0, forcing=target.forcing, seed=target.seed)
        om = workloads.build(s, oracle)
        u, v, w = S.initial_fields(target)
        om.initialize(vel1=u, vel2=v, vel3=w)
        om.evolve(20 * DT, DT)
        _close(target.result, om.state, TRAJ_TOL)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_elastic_server_request_same_alone_and_in_mix(oracle, BLD, precision, tol):
    """Pools created and released against the HBM budget (ElasticServer), requests
    initialised on the device: a request gives the same result alone and among
    concurrent requests, and (FP64) the oracle's trajectory from the same seeded
    field.  The budget holds two pools, so pools are released and re-made."""
    from BoundaryLayerDynamics import serving as S
    from BoundaryLayerDynamics import workloads
    sizes = ((16, 8), (24, 12))

    def server():
        def factory(size, n):
            return workloads.build(S.spec_for(size), BLD, precision=precision, members=n)
        return S.ElasticServer(factory, {(16, 8): 3, (24, 12): 2}, {(16, 8): 10, (24, 12): 10}, budget=20, dt=DT,
                               tick=5, keep_results=True)

    def requests():
        return S.make_requests(12, rate=2000.0, seed=11, sizes=sizes, probs=(0.5, 0.5), steps=20, materialize=False)

    mix = requests()
    srv = server()
    st = srv.run(mix)
    assert st["completed"] == 12 and st["peak_resident_bytes"] <= 20
    target = mix[7]
    alone = [r for r in requests() if r.rid == target.rid]
    alone[0].arrival = 0.0
    assert server().run(alone)["completed"] == 1
    _close(target.result, alone[0].result, tol)
    if precision == "fp64":
        s = S.spec_for(target.size, z0=target.z0, forcing=target.forcing, seed=target.seed)
        om = workloads.build(s, oracle)
        u, v, w = workloads.seeded_initial_fields(s, target.seed)
        om.initialize(vel1=u, vel2=v, vel3=w)
        om.evolve(20 * DT, DT)
        _close(target.result, om.state, TRAJ_TOL)
