"""GPU parity: the CUDA engine (through its C ABI) against the FP64 oracle.

Bars (plain FP64 form): rates and projections within 1e-12 relative L2 per
field; trajectories within 1e-9 relative L2 after 100 steps.  Mixed form:
within 1e-5 relative.  Inputs are identical spectral bytes for both sides.
"""

import math

import numpy as np
import pytest

from conftest import approx, rel_l2

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
TRAJ_TOL = 1e-9


@pytest.fixture(scope="module")
def BLD():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as B
    return B


def _pair(oracle, BLD, resolution, dom_fn, procs_fn, **kw):
    om = oracle.Model(resolution, dom_fn(oracle), procs_fn(oracle))
    gm = BLD.Model(resolution, dom_fn(BLD), procs_fn(BLD), **kw)
    return om, gm


def _random_state(om, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    st = {}
    for f in om.fields:
        shape = om.state[f].shape
        # decaying spectrum, so the physical fields stay O(1)
        k1 = np.arange(shape[2])[None, None, :]
        k2 = np.abs(om.grid.wavenumbers(2))[None, :, None]
        amp = scale / (1.0 + k1 ** 2 + k2 ** 2)
        st[f] = amp * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    return st


def _ic_state(om, spec, seed=None):
    from BoundaryLayerDynamics import workloads
    u, v, w = workloads.initial_fields(spec, seed)
    om.initialize(vel1=u, vel2=v, vel3=w)
    return {f: om.state[f].copy() for f in om.fields}


# ------------------------------------------------------------------- model builders
def _dns(api, size=(4 * math.pi, 2 * math.pi, 2.0)):
    return api.Domain(size, api.SmoothWall(), api.SmoothWall())


def _les(api, size=(2 * math.pi, math.pi, 1.0)):
    return api.Domain(size, api.RoughWall(1e-4), api.FreeSlipBoundary())


CASES = {
    "dns_16x16x8": ((16, 16, 8), _dns, lambda a: a.incompressible_flow(1 / 180, constant_forcing=1)),
    "dns_12x16x5": ((12, 16, 5), _dns, lambda a: a.incompressible_flow(0.01, constant_forcing=(1, 0.5))),
    "les_16x16x8": ((16, 16, 8), _les, lambda a: a.incompressible_flow(
        1e-5, constant_forcing=1, sgs_model=a.StaticSmagorinskyModel())),
    "les_24x18x7_nodamp": ((24, 18, 7), lambda a: a.Domain((2.0, 1.5, 1.0), a.RoughWall(1e-3), a.RoughWall(2e-3)),
                           lambda a: [a.StaticSmagorinskyModel(Cs=0.13, wall_damping=False), a.MolecularDiffusion("vel1", 1e-3)]),
    "adv_nodealias_freeslip": ((16, 16, 6), lambda a: a.Domain((1, 1, 1), a.FreeSlipBoundary(), a.FreeSlipBoundary()),
                               lambda a: [a.MomentumAdvection(dealiasing=None), a.Pressure()]),
    "stretched_dns": ((16, 12, 9), lambda a: a.Domain((2.0, 2.0, 1.0), a.SmoothWall(), a.SmoothWall(), a.SinusoidalMapping(0.9)),
                      lambda a: a.incompressible_flow(0.05, constant_flux=(1.0, 0.3))),
    "diffusion_custom": ((12, 18, 6), lambda a: a.Domain(
        (2 * math.pi, 2 * math.pi, 1.0),
        a.CustomBoundary(vel1=("neumann", 1.3), vel2=("dirichlet", 0.4), vel3=("dirichlet", 0.2)),
        a.CustomBoundary(vel1=("neumann", -0.7), vel2=("dirichlet", 0.4), vel3=("dirichlet", 0.2))),
        lambda a: [a.MolecularDiffusion(v, 1e-2) for v in ("vel1", "vel2", "vel3")] + [a.ConstantSource("vel2", 0.7)]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_rates_parity(oracle, BLD, case):
    res, dom, procs = CASES[case]
    om, gm = _pair(oracle, BLD, res, dom, procs)
    st = _random_state(om, seed=hash(case) % 1000)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        assert rel_l2(got[f], ref[f]) < RHS_TOL, (f, rel_l2(got[f], ref[f]))


@pytest.mark.parametrize("case", sorted(CASES))
def test_projection_parity(oracle, BLD, case):
    res, dom, procs = CASES[case]
    om, gm = _pair(oracle, BLD, res, dom, procs)
    st = _random_state(om, seed=7)
    a = {f: v.copy() for f, v in st.items()}
    b = {f: v.copy() for f, v in st.items()}
    om.apply_projections(a)
    gm.apply_projections(b)
    for f in om.fields:
        assert rel_l2(b[f], a[f]) < RHS_TOL, (f, rel_l2(b[f], a[f]))


def test_pressure_nonzero_w_boundary(oracle, BLD):
    """test/pressure_test.jl:40-74 through the engine: w = bc3 everywhere after projection."""
    bc3 = 0.5700899056030746
    dom = lambda a: a.Domain((2 * math.pi, 2 * math.pi, 1.0),
                             a.CustomBoundary(vel1="dirichlet", vel2="dirichlet", vel3=("dirichlet", bc3)),
                             a.CustomBoundary(vel1="dirichlet", vel2="dirichlet", vel3=("dirichlet", bc3)))
    om, gm = _pair(oracle, BLD, (4, 4, 16), dom, lambda a: [a.Pressure()])
    BLD.initialize(gm, vel1=lambda x, y, z: 1 + np.sin(x))
    st = gm.state
    gm.apply_projections(st)
    gm.set_state(st)
    assert approx(gm["vel1"], np.ones(gm["vel1"].shape))
    BLD.initialize(gm)
    st = gm.state
    gm.apply_projections(st)
    gm.set_state(st)
    assert approx(gm["vel3"], bc3 * np.ones(gm["vel3"].shape))


def test_rates_parity_les64(oracle, BLD):
    """The half-channel LES workload at full size (64^2 x 32), seeded log-law IC."""
    from BoundaryLayerDynamics import workloads
    spec = workloads.CONFIGS["les64"]
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    st = _ic_state(om, spec)
    om.apply_projections(st)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        assert rel_l2(got[f], ref[f]) < RHS_TOL, (f, rel_l2(got[f], ref[f]))


def test_rates_parity_dns192(oracle, BLD):
    """The closed-channel DNS at full size (192^2 x 96): oracle at the reference's 286^2
    padding, engine at 288^2 (both exact for quadratic products)."""
    from BoundaryLayerDynamics import workloads
    spec = workloads.CONFIGS["dns192"]
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    assert (gm.info.adv_ref_p1, gm.info.adv_p1) == (286, 288)
    st = _ic_state(om, spec)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        assert rel_l2(got[f], ref[f]) < RHS_TOL, (f, rel_l2(got[f], ref[f]))


@pytest.mark.parametrize("method", ["SSPRK33", "SSPRK22", "Euler", "AB2"])
def test_trajectory_parity(oracle, BLD, method):
    """100 steps through evolve! from identical spectral bytes; <= 1e-9 relative."""
    from BoundaryLayerDynamics import workloads
    spec = workloads.les_spec(16, 8, (2 * math.pi, math.pi, 1.0), steps=100)
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    st = _ic_state(om, spec)
    gm.set_state(st)
    dt = 1e-3
    om.evolve(100 * dt, dt, method=getattr(oracle, method))
    gm.evolve(100 * dt, dt, method=getattr(BLD, method))
    got = gm.state
    for f in om.fields:
        assert rel_l2(got[f], om.state[f]) < TRAJ_TOL, (f, rel_l2(got[f], om.state[f]))


@pytest.mark.parametrize("method", ["SSPRK33", "SSPRK22"])
@pytest.mark.parametrize("case", ["dns_16x16x8", "les_16x16x8", "stretched_dns", "les_24x18x7_nodamp"])
def test_stage_fusion_matches_unfused(oracle, BLD, case, method):
    """The SSP-RK stage update formed in the forward y pass, with the steps of one
    call chained (the trailing right-hand side forms the next step's Euler stage),
    against the same 20 steps with the update in the projection
    (BLD_NO_STAGE_FUSION=1) and against one step per call (no chaining): 1e-12
    between the engine paths, and the oracle's trajectory tolerance."""
    import os
    res, dom, procs = CASES[case]
    om = oracle.Model(res, dom(oracle), procs(oracle))
    st = _random_state(om, seed=len(case), scale=2.0)
    om.apply_projections(st)
    meth = getattr(BLD, method)
    runs = []
    for off, per_call in (("0", 20), ("1", 20), ("0", 1)):
        old = os.environ.get("BLD_NO_STAGE_FUSION")
        os.environ["BLD_NO_STAGE_FUSION"] = off
        try:
            gm = BLD.Model(res, dom(BLD), procs(BLD))
            gm.set_state(st)
            if per_call == 20:
                gm.evolve(20 * 1e-3, 1e-3, method=meth)
            else:
                gm.evolve(1e-3, 1e-3, method=meth)
                for _ in range(19):
                    gm.step(1, 1e-3, meth)
            runs.append(gm.state)
        finally:
            if old is None:
                del os.environ["BLD_NO_STAGE_FUSION"]
            else:
                os.environ["BLD_NO_STAGE_FUSION"] = old
    om.state.update({f: v.copy() for f, v in st.items()})
    om.evolve(20 * 1e-3, 1e-3, method=getattr(oracle, method))
    for f in om.fields:
        for r in runs[1:]:
            assert rel_l2(runs[0][f], r[f]) < 1e-12, (f, rel_l2(runs[0][f], r[f]))
        assert rel_l2(runs[0][f], om.state[f]) < TRAJ_TOL, (f, rel_l2(runs[0][f], om.state[f]))


def test_trajectory_parity_dns(oracle, BLD):
    spec = dict(kind="dns", resolution=(24, 24, 12), size=(4 * math.pi, 2 * math.pi, 2.0), lower=("smooth",),
                upper=("smooth",), nu=1 / 180, forcing=1.0, sgs=None, dt=1e-4, steps=100, seed=5)
    from BoundaryLayerDynamics import workloads
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD)
    st = _ic_state(om, spec)
    gm.set_state(st)
    om.evolve(100 * 1e-4, 1e-4)
    gm.evolve(100 * 1e-4, 1e-4)
    got = gm.state
    for f in om.fields:
        assert rel_l2(got[f], om.state[f]) < TRAJ_TOL, (f, rel_l2(got[f], om.state[f]))


def test_physical_transforms(oracle, BLD):
    """initialize! and getindex at the default size against the oracle's set_field!/get_field."""
    res, dom, procs = CASES["les_16x16x8"]
    om, gm = _pair(oracle, BLD, res, dom, procs)
    rng = np.random.default_rng(11)
    vals = {f: rng.standard_normal((om.grid.nz(oracle.NODES[f]), 16, 16)) for f in ("vel1", "vel2", "vel3")}
    om.initialize(**vals)
    BLD.initialize(gm, **vals)
    for f in om.fields:
        assert rel_l2(gm.state[f], om.state[f]) < RHS_TOL
        assert rel_l2(gm[f], om[f]) < RHS_TOL


def test_mixed_precision_rates(oracle, BLD):
    from BoundaryLayerDynamics import workloads
    spec = workloads.les_spec(32, 16, (2 * math.pi, math.pi, 1.0))
    om = workloads.build(spec, oracle)
    gm = workloads.build(spec, BLD, precision="mixed")
    st = _ic_state(om, spec)
    om.apply_projections(st)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-5, (f, e)


def test_divergence_flag(oracle, BLD):
    """A non-finite rate raises 'The simulation has diverged.' (src/BoundaryLayerDynamics.jl:155-157)."""
    res, dom, procs = CASES["dns_16x16x8"]
    om, gm = _pair(oracle, BLD, res, dom, procs)
    st = _random_state(om, seed=3)
    st["vel2"][2, 3, 1] = np.nan
    with pytest.raises(BLD.DivergenceError, match="diverged"):
        gm.compute_rates(st)
    st["vel2"][2, 3, 1] = 0.0
    gm.compute_rates(st)  # the flag is cleared after being reported


def test_ensemble_members_match_single(oracle, BLD):
    """Members with their own Cs, roughness and forcing equal single-member models."""
    from BoundaryLayerDynamics import workloads
    spec = workloads.les_spec(16, 8, (2 * math.pi, math.pi, 1.0))
    cs = np.array([0.08, 0.12, 0.16])
    z0 = np.array([1e-5, 1e-4, 1e-3])
    forcing = np.array([1.0, 0.5, 2.0])
    ens = workloads.build(spec, BLD, members=3, member_cs=cs, member_z0=z0, member_forcing=forcing)
    om = workloads.build(spec, oracle)
    base = _ic_state(om, spec)
    for m in range(3):
        ens.set_state({f: base[f] * (1 + 0.1 * m) for f in base}, member=m)
    ens.evolve(10 * 1e-3, 1e-3)
    for m in range(3):
        s = dict(spec, lower=("rough", float(z0[m])), sgs=dict(Cs=float(cs[m])), forcing=float(forcing[m]))
        single = workloads.build(s, BLD)
        single.set_state({f: base[f] * (1 + 0.1 * m) for f in base})
        single.evolve(10 * 1e-3, 1e-3)
        a, b = ens.get_state(m), single.state
        for f in a:
            assert rel_l2(a[f], b[f]) < 1e-14, (m, f, rel_l2(a[f], b[f]))


LDLT_TOL = 1e-13   # the segmented solve reassociates the recurrences; diagonally dominant systems


@pytest.mark.parametrize("n,nsys", [(1, 5), (2, 33), (3, 1), (7, 100), (24, 1000), (96, 517), (255, 64),
                                    (256, 300), (257, 300), (511, 40), (512, 77), (700, 20), (1024, 33)])
@pytest.mark.parametrize("kind", ["complex", "real"])
def test_ldlt_solve_device(oracle, BLD, n, nsys, kind):
    """The standalone batched LDL^T kernel (segmented) against the oracle's ldlt_solve,
    including ragged sizes (n not a multiple of the segment length, nsys not a
    multiple of the systems per block)."""
    import torch
    from BoundaryLayerDynamics import _capi
    lib = _capi.load()
    rng = np.random.default_rng(n * 1000 + nsys)
    diag = -2.0 - rng.random((nsys, n))
    off = 0.5 + 0.3 * rng.random(max(n - 1, 1))[: n - 1]
    gam = oracle.ldlt_factor(diag, off)                    # (nsys, n)
    rhs = rng.standard_normal((n, nsys))
    if kind == "complex":
        rhs = rhs + 1j * rng.standard_normal((n, nsys))
    ref = oracle.ldlt_solve(gam, off, rhs.copy())
    g_d = torch.tensor(np.ascontiguousarray(gam.T), device="cuda")
    b_d = torch.tensor(np.concatenate([off, [0.0]]), device="cuda")
    r_d = torch.tensor(rhs, device="cuda")
    fn = lib.bld_ldlt_solve_device if kind == "complex" else lib.bld_ldlt_solve_real_device
    _capi.check(fn(g_d.data_ptr(), b_d.data_ptr(), r_d.data_ptr(), nsys, n, None))
    torch.cuda.synchronize()
    assert rel_l2(r_d.cpu().numpy(), ref) < LDLT_TOL


def test_ldlt_solve_rejects_bad_sizes(BLD):
    from BoundaryLayerDynamics import _capi
    lib = _capi.load()
    assert lib.bld_ldlt_solve_device(1, 1, 1, 10, 1025, None) == _capi.BLD_ERR_ARGUMENT
    assert lib.bld_ldlt_solve_real_device(1, 1, 1, 0, 10, None) == _capi.BLD_ERR_ARGUMENT
