"""Physical sizes with the prime factors 5 and 7 against the oracle.

The reference transforms at any size FFTW plans (src/physical_space.jl:14-21,
42-61): Smagorinsky spaces without dealiasing use exactly 2k + 2 points
(src/physical_space.jl:49-56), and any process may ask for explicit sizes
(`dealiasing = (N1, N2)`).  The engine's block Stockham kernels carry radix 5,
7, 10, 14 and 15 codelets besides the 2^a 3^b ones, so these sizes run on the
GPU as well; the checks are the usual ones (rates and a short trajectory at
1e-12 / 1e-10 in FP64, 1e-5 in the mixed form).
"""

import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def BLD():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as B
    return B


def _les(api, res, precision=None):
    dom = api.Domain((2 * math.pi, math.pi, 1.0), api.RoughWall(1e-4), api.FreeSlipBoundary())
    procs = api.incompressible_flow(1e-5, constant_forcing=1, sgs_model=api.StaticSmagorinskyModel())
    kw = {} if precision is None else dict(precision=precision)
    return api.Model(res, dom, procs, **kw)


def _dns_explicit(api, res, sizes, precision=None):
    dom = api.Domain((4 * math.pi, 2 * math.pi, 2.0), api.SmoothWall(), api.SmoothWall())
    procs = ([api.MomentumAdvection(dealiasing=sizes)] +
             [api.MolecularDiffusion(f, 1 / 180) for f in ("vel1", "vel2", "vel3")] +
             [api.Pressure(), api.ConstantSource("vel1", 1.0)])
    kw = {} if precision is None else dict(precision=precision)
    return api.Model(res, dom, procs, **kw)


def _state(om, seed):
    rng = np.random.default_rng(seed)
    st = {}
    for f in om.fields:
        shape = om.state[f].shape
        k1 = np.arange(shape[2])[None, None, :]
        k2 = np.abs(om.grid.wavenumbers(2))[None, :, None]
        st[f] = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / (1.0 + k1 ** 2 + k2 ** 2)
    om.apply_projections(st)
    return st


# (resolution, physical sizes of the Smagorinsky space): 80 = 16 x 5,
# 100 = 10 x 10, 70 = 14 x 5, 56 = 8 x 7, 42 = 14 x 3
LES_CASES = [((80, 80, 8), (80, 80)), ((100, 70, 6), (100, 70)), ((56, 42, 6), (56, 42))]


@pytest.mark.parametrize("res,P", LES_CASES)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_les_sgs_sizes_with_5_and_7(oracle, BLD, res, P, precision, tol):
    om = _les(oracle, res)
    gm = _les(BLD, res, precision)
    assert (gm.info.sgs_p1, gm.info.sgs_p2) == P, (gm.info.sgs_p1, gm.info.sgs_p2)
    assert gm.kernels()["sgs"]["x"].startswith("k_sgs_x<"), gm.kernels()
    st = _state(om, seed=sum(res))
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (res, precision, f, e)


@pytest.mark.parametrize("sizes", [(112, 98), (140, 150)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_explicit_dealiasing_sizes_with_5_and_7(oracle, BLD, sizes, precision, tol):
    res = (64, 48, 6)
    om = _dns_explicit(oracle, res, sizes)
    gm = _dns_explicit(BLD, res, sizes, precision)
    assert (gm.info.adv_p1, gm.info.adv_p2) == sizes
    st = _state(om, seed=sum(sizes))
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (sizes, precision, f, e)


def test_les_80_trajectory(oracle, BLD):
    """Ten SSP-RK33 steps of the 80 x 80 x 8 LES (Smagorinsky space 80 x 80)."""
    res = (80, 80, 8)
    om = _les(oracle, res)
    gm = _les(BLD, res)
    st = _state(om, seed=3)
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    gm.evolve(10 * 1e-4, 1e-4)
    om.evolve(10 * 1e-4, 1e-4)
    for f in om.fields:
        e = rel_l2(gm.state[f], om.state[f])
        assert e < 1e-10, (f, e)


def test_unsupported_prime_factor_rejected(BLD):
    """A Smagorinsky space of 2 x 11 x 11 points (resolution 242) has no codelet
    plan: the model is rejected with an error instead of running."""
    with pytest.raises(Exception) as err:
        _les(BLD, (242, 16, 4))
    assert "physical-domain size 242" in str(err.value), err.value
