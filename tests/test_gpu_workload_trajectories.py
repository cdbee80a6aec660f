"""GPU trajectories of the benchmark workloads at full size against the FP64 oracle.

* Half-channel LES 64x64x32 (2pi x pi x 1, RoughWall(1e-4) / FreeSlipBoundary,
  StaticSmagorinskyModel(Cs=0.1), unit forcing, seeded log-law + 10 % noise):
  100 SSP-RK33 steps of dt = 1e-4 through evolve! in the plain FP64 form,
  <= 1e-9 relative L2 per field (src/ODEMethods.jl:147-166, test/les_test.jl:50-72).
* The same LES over 1000 steps in the mixed form (FP32 transforms, products and
  SGS; FP64 state, stage updates and pressure solve): relative velocity error
  against the FP64 oracle <= 1e-5, and the divergence of the final state at the
  oracle's level (the FP64 projection leaves it at rounding).
* Closed-channel DNS 192x192x96 (4pi x 2pi x 2, nu = 1/180, seeded laminar
  profile + Gaussian noise): 10 SSP-RK33 steps in the plain form, engine at the
  288^2 padding against the oracle at the reference's 286^2, <= 1e-9.

The oracle runs on all host cores (pocketfft workers); the LES trajectory is
computed once and shared by the FP64 and mixed checks.
"""

import math
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TRAJ_TOL = 1e-9
MIXED_TOL = 1e-5


@pytest.fixture(scope="module")
def BLD():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as B
    return B


@pytest.fixture(scope="module")
def fast_oracle(oracle):
    oracle.set_fft_workers(os.cpu_count() or 1)
    yield oracle
    oracle.set_fft_workers(1)


def _initial_state(om, spec):
    from BoundaryLayerDynamics import workloads
    u, v, w = workloads.initial_fields(spec)
    om.initialize(vel1=u, vel2=v, vel3=w)
    return {f: om.state[f].copy() for f in om.fields}


def divergence_max(state, spec, K1, k2max, n3):
    """max |D1 u + D2 v + d3 w| over all modes of a state on an unmapped grid with
    w = 0 at both walls (the divergence the pressure projection removes,
    src/processes/pressure.jl:368-378)."""
    L1, L2, L3 = spec["size"]
    k1 = np.arange(K1)
    k2 = np.concatenate([np.arange(k2max + 1), np.arange(-k2max, 0)])
    D1 = (1j * k1 * 2 * math.pi / L1)[None, None, :]
    D2 = (1j * k2 * 2 * math.pi / L2)[None, :, None]
    w = state["vel3"]
    zero = np.zeros_like(w[:1])
    wext = np.concatenate([zero, w, zero])
    div = D1 * state["vel1"] + D2 * state["vel2"] + (wext[1:] - wext[:-1]) * (n3 / L3)
    return float(np.abs(div).max())


def _rel_velocity(a, b):
    num = sum(np.linalg.norm((a[f] - b[f]).ravel()) ** 2 for f in b)
    den = sum(np.linalg.norm(b[f].ravel()) ** 2 for f in b)
    return math.sqrt(num / den)


@pytest.fixture(scope="module")
def les64_oracle(fast_oracle):
    """Initial state and the oracle's states after 100 and 1000 SSP-RK33 steps."""
    from BoundaryLayerDynamics import workloads
    spec = workloads.CONFIGS["les64"]
    om = workloads.build(spec, fast_oracle)
    st0 = _initial_state(om, spec)
    dt = spec["dt"]
    om.evolve(100 * dt, dt)
    s100 = {f: om.state[f].copy() for f in om.fields}
    # continuing from the checkpoint re-applies one (idempotent) projection and
    # the rates at the new time, as step_to! does between checkpoints
    om.evolve(900 * dt, dt)
    s1000 = {f: om.state[f].copy() for f in om.fields}
    return spec, st0, s100, s1000


def test_les64_100_steps_fp64(BLD, les64_oracle):
    from BoundaryLayerDynamics import workloads
    spec, st0, s100, _ = les64_oracle
    gm = workloads.build(spec, BLD)
    gm.set_state(st0)
    dt = spec["dt"]
    gm.evolve(100 * dt, dt)
    got = gm.state
    for f in s100:
        e = rel_l2(got[f], s100[f])
        assert e < TRAJ_TOL, (f, e)


def test_les64_1000_steps_mixed_against_fp64_oracle(BLD, les64_oracle):
    from BoundaryLayerDynamics import workloads
    spec, st0, s100, s1000 = les64_oracle
    gm = workloads.build(spec, BLD, precision="mixed")
    gm.set_state(st0)
    dt = spec["dt"]
    gm.evolve(100 * dt, dt)
    e100 = _rel_velocity(gm.state, s100)
    gm.evolve(900 * dt, dt)
    got = gm.state
    e1000 = _rel_velocity(got, s1000)
    n3 = spec["resolution"][2]
    K1, K2 = got["vel1"].shape[2], got["vel1"].shape[1]
    div_gpu = divergence_max(got, spec, K1, (K2 - 1) // 2, n3)
    div_ref = divergence_max(s1000, spec, K1, (K2 - 1) // 2, n3)
    scale = max(float(np.abs(s1000[f]).max()) for f in s1000)
    print(f"mixed LES 64^2x32: rel. velocity error {e100:.3e} after 100 steps, {e1000:.3e} after 1000; "
          f"max |div u| {div_gpu:.3e} (oracle {div_ref:.3e}, max |u| {scale:.3g})")
    assert e1000 < MIXED_TOL, e1000
    assert div_gpu < 1e-12 * scale, (div_gpu, div_ref)


def test_dns192_10_steps_fp64(BLD, fast_oracle):
    from BoundaryLayerDynamics import workloads
    spec = workloads.CONFIGS["dns192"]
    om = workloads.build(spec, fast_oracle)
    gm = workloads.build(spec, BLD)
    assert (gm.info.adv_ref_p1, gm.info.adv_p1) == (286, 288)
    st0 = _initial_state(om, spec)
    gm.set_state(st0)
    dt = spec["dt"]
    om.evolve(10 * dt, dt)
    gm.evolve(10 * dt, dt)
    got = gm.state
    for f in om.fields:
        e = rel_l2(got[f], om.state[f])
        assert e < TRAJ_TOL, (f, e)
