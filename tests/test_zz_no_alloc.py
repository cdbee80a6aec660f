"""The allocation-free pressure projection, bld_project_noalloc.

Some callers cannot let a library call cudaMalloc: their device memory belongs
to a host framework's pool (for example a Julia CuArray pool, or an
application embedding the engine under a fixed memory budget), so every buffer
must come from them.  bld_project_noalloc takes all inputs and outputs from the
caller and keeps its only scratch in a fixed array inside the library.  The GPU
test checks it against the regular projection entry point
(bld_apply_projections) on two calls in a row, within the 1e-12 relative
tolerance of the other parity tests, with w = 0 at smooth walls and with an
equal non-zero Dirichlet w at both boundaries (the divergence's wall terms of
the mean mode).  The test allocates its own buffers with torch; the entry point
itself allocates nothing.  The argument checks happen before any device work,
so they run on the CPU too.
"""

import math

import numpy as np
import pytest

from conftest import rel_l2

TOL = 1e-12
W_WALL = 0.37


def _smooth(api):
    return api.Domain((2.0, 1.5, 1.0), api.SmoothWall(), api.SmoothWall(), api.SinusoidalMapping(0.8))


def _moving(api):
    b = lambda: api.CustomBoundary(vel1="dirichlet", vel2="dirichlet", vel3=("dirichlet", W_WALL))
    return api.Domain((2.0, 1.5, 1.0), b(), b())


@pytest.mark.gpu
@pytest.mark.parametrize("domain,w_wall", [(_smooth, 0.0), (_moving, W_WALL)], ids=["smooth", "w_wall"])
def test_project_noalloc_matches_apply_projections(oracle, domain, w_wall):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as BLD
    from BoundaryLayerDynamics import _capi

    lib = _capi.load()
    res = (24, 18, 10)
    om = oracle.Model(res, domain(oracle), [oracle.Pressure()])
    gm = BLD.Model(res, domain(BLD), [BLD.Pressure()])
    press = om.processes[0]
    g = om.grid
    K1, K2, n3 = g.K1, g.K2, g.n3global
    # the Pressure process tables, in the layout the entry point documents
    gamma = np.ascontiguousarray(press.gamma.reshape(K2 * K1, n3).T)          # [n3][F]
    alpha_c = oracle.dx3factors(om.domain, g, "C")
    alpha_i = oracle.dx3factors(om.domain, g, "I")
    d1 = g.wavenumbers(1) * (2 * math.pi / om.domain.hsize[0])
    d2 = g.wavenumbers(2) * (2 * math.pi / om.domain.hsize[1])
    dev = {k: torch.tensor(np.ascontiguousarray(v, dtype=np.float64), device="cuda")
           for k, v in dict(gamma=gamma, ac=alpha_c, ai=alpha_i, d1=d1, d2=d2).items()}
    rng = np.random.default_rng(20)
    for call in range(2):
        st = {f: rng.standard_normal(gm.zeros(f).shape) + 1j * rng.standard_normal(gm.zeros(f).shape)
              for f in ("vel1", "vel2", "vel3")}
        ref = {f: v.copy() for f, v in st.items()}
        gm.apply_projections(ref)                       # the existing entry point
        packed = np.concatenate([st[f].ravel() for f in ("vel1", "vel2", "vel3")])
        d_state = torch.tensor(packed, device="cuda")
        status = lib.bld_project_noalloc(g.k1max, g.k2max, n3, dev["gamma"].data_ptr(), dev["ac"].data_ptr(),
                                         dev["ai"].data_ptr(), dev["d1"].data_ptr(), dev["d2"].data_ptr(),
                                         w_wall, w_wall, d_state.data_ptr(), None)
        _capi.check(status)
        torch.cuda.synchronize()
        out = d_state.cpu().numpy()
        nc = n3 * K2 * K1
        got = {"vel1": out[:nc], "vel2": out[nc:2 * nc], "vel3": out[2 * nc:]}
        for f in got:
            e = rel_l2(got[f], ref[f].ravel())
            assert e < TOL, (call, f, e)


def _lib():
    import BoundaryLayerDynamics as BLD  # noqa: F401
    from BoundaryLayerDynamics import _capi
    return _capi.load(), _capi


DUMMY = 1  # non-null placeholders: every check below fires before any device work


def test_project_noalloc_rejects_sizes_above_its_scratch():
    lib, _capi = _lib()
    # 96 x 191 modes x 96 layers = 1.76e6 complex values > 2^20
    status = lib.bld_project_noalloc(95, 95, 96, DUMMY, DUMMY, DUMMY, DUMMY, DUMMY, 0.0, 0.0, DUMMY, None)
    assert status == _capi.BLD_ERR_INVALID_CONFIG
    with pytest.raises(_capi.BldError, match="exceeds the fixed scratch"):
        _capi.check(status)
    # sizes whose 32-bit product would wrap around are rejected, not wrapped
    status = lib.bld_project_noalloc(2**30, 2**30, 3, DUMMY, DUMMY, DUMMY, DUMMY, DUMMY, 0.0, 0.0, DUMMY, None)
    assert status == _capi.BLD_ERR_INVALID_CONFIG


def test_project_noalloc_rejects_unequal_wall_velocities():
    """src/processes/pressure.jl:357: error("The mean flow must be equal at both vertical boundaries.")"""
    lib, _capi = _lib()
    status = lib.bld_project_noalloc(4, 4, 6, DUMMY, DUMMY, DUMMY, DUMMY, DUMMY, 0.1, 0.2, DUMMY, None)
    assert status == _capi.BLD_ERR_UNSUPPORTED_BC
    with pytest.raises(_capi.BldError, match="mean flow must be equal"):
        _capi.check(status)
