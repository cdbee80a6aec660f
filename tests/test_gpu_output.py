"""Output on the device: centered transforms, Snapshots and MeanProfiles.

* get_field/set_field with the half-grid-point shift against the oracle (1e-12);
* evolve(..., output=[Snapshots]) writes the reference's CBD layout at the
  snapshot times with the oracle's trajectory values (1e-9), and
  initialize(model, path) reads a snapshot back into the same state (1e-12);
* evolve(..., output=[MeanProfiles]) integrates the horizontal means on the
  device and matches the oracle's per-step trapezoidal sums (1e-9).
"""

import math
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

DT = 1e-3


@pytest.fixture(scope="module")
def BLD():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as B
    return B


def _spec():
    from BoundaryLayerDynamics import workloads
    return workloads.les_spec(16, 8, (2 * math.pi, math.pi, 1.0))


def _pair(oracle, BLD, seed=3):
    from BoundaryLayerDynamics import workloads
    spec = _spec()
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    u, v, w = workloads.initial_fields(spec, seed)
    om.initialize(vel1=u, vel2=v, vel3=w)
    gm.set_state({f: om.state[f].copy() for f in om.fields})
    return om, gm


def test_centered_transforms(oracle, BLD):
    om, gm = _pair(oracle, BLD)
    for f in om.fields:
        ref = om.get_field(f, centered=True)
        got = gm.get_field(f, centered=True)
        assert rel_l2(got, ref) < 1e-12, f
    pd = om.get_field("vel2", centered=True) * 1.5
    om.set_field("vel2", pd, centered=True)
    gm.set_field("vel2", pd, centered=True)
    assert rel_l2(gm.state["vel2"], om.state["vel2"]) < 1e-12


def test_snapshots_and_restart(oracle, BLD, tmp_path):
    from BoundaryLayerDynamics import cbd
    om, gm = _pair(oracle, BLD)
    path = str(tmp_path / "snapshots")
    snaps = BLD.Snapshots(frequency=4 * DT, path=path)
    gm.evolve(10 * DT, DT, output=[snaps])
    assert sorted(os.listdir(path)) == ["state-001", "state-002"]
    # oracle trajectory up to the second snapshot time
    om.evolve(8 * DT, DT)
    for f in om.fields:
        xmin, xmax, x1, x2, x3, data = cbd.readcbd(os.path.join(path, "state-002", f"{f}.cbd"))
        assert rel_l2(data, om.get_field(f, centered=True)) < 1e-9, f
        assert x1[0] > 0                                          # centred coordinates
        assert np.allclose(x3, gm.coordinates(f)[2])
    # initialize!(model, path) from the snapshot
    gm2 = BLD.Model(gm.resolution, gm.domain, gm.processes)
    BLD.initialize(gm2, os.path.join(path, "state-002"))
    for f in om.fields:
        assert rel_l2(gm2.state[f][:, :, 1:], om.state[f][:, :, 1:]) < 1e-11, f


def test_mean_profiles_on_device(oracle, BLD, tmp_path):
    DT = 1.0 / 1024   # a binary fraction, so that the step-by-step oracle times are exact
    om, gm = _pair(oracle, BLD, seed=5)
    path = str(tmp_path / "profiles")
    mp = BLD.MeanProfiles(path=path, output_frequency=5 * DT)
    gm.evolve(10 * DT, DT, output=[mp])
    assert [os.path.basename(f) for f in mp.files] == ["profiles-01.npz", "profiles-02.npz"]
    # oracle: the projected initial state is the first sample, then one per step
    ref = oracle.MeanProfiles(om.grid.n3global, 0.0)
    om.apply_projections(om.state)
    ref.sample_state(om.state)
    got = []
    for k in range(1, 11):
        om.evolve(((k - 1) * DT, k * DT), DT)
        ref.step(om.state, k * DT)
        if k % 5 == 0:
            got.append(ref.averages())
            ref = oracle.MeanProfiles(om.grid.n3global, k * DT)
            ref.sample_state(om.state)
    for fn, want in zip(mp.files, got):
        d = np.load(fn)
        assert int(d["intervals"]) == 5
        for f in ("vel1", "vel2", "vel3"):
            assert d[f].shape == want[f].shape
            assert np.allclose(d[f], want[f], rtol=1e-9, atol=1e-12), (fn, f)


@pytest.mark.parametrize("case", ["les", "dns"])
def test_progress_stats_match_oracle(oracle, BLD, case):
    """ProgressMonitor statistics from the device (src/logging.jl:215-276) against
    the oracle's restatement: mean velocity, mean and turbulent kinetic energy
    (Parseval on the device, physical means in the oracle), the advective time
    scale from max |w| on the largest physical grid, and the wall-model stresses
    of the rough wall (1e-12 relative; LES 32^2x16 has the same grids on both
    sides: advection 48^2, SGS 32^2).  The DNS case (32^2x12: advection 48^2)
    also checks the smooth-wall model without wall stresses."""
    from BoundaryLayerDynamics import workloads
    if case == "les":
        spec = workloads.les_spec(32, 16, (2 * math.pi, math.pi, 1.0))
    else:
        spec = dict(kind="dns", resolution=(32, 32, 12), size=(4 * math.pi, 2 * math.pi, 2.0), lower=("smooth",),
                    upper=("smooth",), nu=1 / 180, forcing=1.0, sgs=None, dt=1e-4, steps=10, seed=5)
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    u, v, w = workloads.initial_fields(spec)
    om.initialize(vel1=u, vel2=v, vel3=w)
    st = {f: om.state[f].copy() for f in om.fields}
    om.apply_projections(st)
    gm.set_state(st)
    ref = oracle.progress_stats(om, st, tstep=1e-4)
    got = gm.progress(tstep=1e-4)
    assert set(got) == set(ref), (sorted(got), sorted(ref))
    for k, r in ref.items():
        rv, gv = np.atleast_1d(np.asarray(r, float)), np.atleast_1d(np.asarray(got[k], float))
        scale = max(np.abs(rv).max(), 1e-300)
        assert np.abs(gv - rv).max() <= 1e-12 * scale, (k, gv, rv)


def test_progress_monitor_module(BLD):
    """evolve(..., output=[ProgressMonitor]) reports at its checks and at the end
    with the device statistics."""
    import io
    from BoundaryLayerDynamics import workloads
    spec = workloads.les_spec(16, 8, (2 * math.pi, math.pi, 1.0))
    gm = workloads.build(spec, BLD)
    u, v, w = workloads.initial_fields(spec)
    BLD.initialize(gm, vel1=u, vel2=v, vel3=w)
    buf = io.StringIO()
    pm = BLD.ProgressMonitor(frequency=0.0, tstep=DT, checks=4, stream=buf)
    BLD.evolve(gm, 8 * DT, dt=DT, output=[pm])
    times = [t for t, _ in pm.reports]
    assert times[-1] == pytest.approx(8 * DT)
    assert len(times) >= 4
    last = pm.reports[-1][1]
    assert last["Adv. Courant Number"] > 0 and last["Mean KE"] > 0
    assert "Mean Velocity" in buf.getvalue()


@pytest.mark.parametrize("kind", ["les", "dns"])
def test_device_initialization_matches_host_fields(oracle, BLD, kind):
    """initialize! with the seeded workload fields generated on the device
    (bld_init_random_field) against the oracle initialised from the same values
    computed on the host (1e-12)."""
    from BoundaryLayerDynamics import workloads
    spec = (workloads.les_spec(32, 16, (2 * math.pi, math.pi, 1.0)) if kind == "les"
            else workloads.dns_spec(24, 12))
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    u, v, w = workloads.seeded_initial_fields(spec, seed=2024)
    om.initialize(vel1=u, vel2=v, vel3=w)
    workloads.initialize_on_device(spec, gm, seed=2024)
    got = gm.state
    for f in om.fields:
        e = rel_l2(got[f], om.state[f])
        assert e < 1e-12, (f, e)
