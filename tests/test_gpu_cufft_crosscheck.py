"""cuFFT cross-check of the hand-written transforms at P = 64 ... 768.

The engine's right-hand side runs its own sm_100a FFT kernels (inverse y,
x passes with the physical-domain products, forward y).  Here the oracle's FFT
backend (the unnormalised rfft2 / brfft of src/physical_space.jl:222,293) is
swapped for cuFFT through torch.fft on the GPU, and the engine's rates are
compared with that oracle at 1e-12 relative L2 -- the same bar as against the
pocketfft oracle.  The cases cover every physical-domain size the benchmark
workloads use: Smagorinsky spaces at P = 2k+2 = 64, 96, 128, 256, 512 and
advection spaces at the 3/2-rule sizes 96, 144, 192, 288 (engine; cuFFT runs
the reference's 286), 384 and 768.  A few layers suffice: the transforms act
per layer.  cuFFT and pocketfft also agree with each other to rounding.
"""

import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def BLD():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as B
    return B


@pytest.fixture
def cufft_oracle(oracle):
    """The oracle with its two FFT entry points running on cuFFT (torch.fft, FP64)."""
    import torch

    def irfft2(h, s):
        return torch.fft.irfft2(torch.from_numpy(np.ascontiguousarray(h)).cuda(), s=s, norm="forward").cpu().numpy()

    def rfft2(x):
        return torch.fft.rfft2(torch.from_numpy(np.ascontiguousarray(x)).cuda(), norm="backward").cpu().numpy()

    saved = (oracle._irfft2_unnormalised, oracle._rfft2_unnormalised)
    oracle._irfft2_unnormalised, oracle._rfft2_unnormalised = irfft2, rfft2
    yield oracle
    oracle._irfft2_unnormalised, oracle._rfft2_unnormalised = saved


def _les(api, n, nz):
    dom = api.Domain((2 * math.pi, math.pi, 1.0), api.RoughWall(1e-4), api.FreeSlipBoundary())
    procs = api.incompressible_flow(1e-5, constant_forcing=1, sgs_model=api.StaticSmagorinskyModel())
    return api.Model((n, n, nz), dom, procs)


def _dns(api, n, nz):
    dom = api.Domain((4 * math.pi, 2 * math.pi, 2.0), api.SmoothWall(), api.SmoothWall())
    return api.Model((n, n, nz), dom, api.incompressible_flow(1 / 180, constant_forcing=1))


def _state(om, seed):
    rng = np.random.default_rng(seed)
    st = {}
    for f in om.fields:
        shape = om.state[f].shape
        k1 = np.arange(shape[2])[None, None, :]
        k2 = np.abs(om.grid.wavenumbers(2))[None, :, None]
        amp = 1.0 / (1.0 + 0.05 * (k1 ** 2 + k2 ** 2))
        st[f] = amp * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    om.apply_projections(st)
    return st


# (builder, n, layers): SGS P = n, advection P = 3/2-rule size of k = n/2 - 1
CASES = {
    "les64": (_les, 64, 6),      # SGS 64, advection 96
    "les96": (_les, 96, 5),      # SGS 96, advection 142 -> 144
    "les128": (_les, 128, 5),    # SGS 128, advection 192
    "dns192": (_dns, 192, 4),    # advection 286 -> 288
    "les256": (_les, 256, 4),    # SGS 256, advection 384
    "les512": (_les, 512, 3),    # SGS 512, advection 768
}


@pytest.mark.parametrize("case", list(CASES))
def test_rates_against_cufft_oracle(BLD, oracle, cufft_oracle, case):
    build, n, nz = CASES[case]
    om = build(cufft_oracle, n, nz)
    gm = build(BLD, n, nz)
    st = _state(om, seed=n)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < TOL, (case, f, e, gm.kernels())


def test_cufft_and_pocketfft_agree(cufft_oracle):
    """The two FFT libraries behind the oracle agree to rounding (DNS at 286^2)."""
    rng = np.random.default_rng(3)
    h = np.fft.rfft2(rng.standard_normal((4, 286, 286)))       # a Hermitian half-spectrum
    a = np.fft.irfft2(h, s=(286, 286), norm="forward")
    b = cufft_oracle._irfft2_unnormalised(h, (286, 286))
    assert rel_l2(b, a) < 1e-14
    x = rng.standard_normal((4, 286, 286))
    assert rel_l2(cufft_oracle._rfft2_unnormalised(x), np.fft.rfft2(x)) < 1e-14
