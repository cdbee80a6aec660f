"""Kernel families the autotuner chooses between, each forced and checked.

The autotuner keeps whichever variant is fastest on the device, so the parity
tests elsewhere exercise only the winners.  Here BLD_X_KERNEL forces the
advection x pass to the warp-per-row kernel (register transforms with lane
shuffles), the block kernel (shared-memory Stockham stages), the block of three
warps per row, its pipelined five-warp form, or the block kernel with warp line
transforms, and each is compared with the oracle at the plain form's 1e-12 and
the mixed form's 1e-5, over every radix the warp kernel is compiled for.
"""

import math
import os

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


def _build(api, res, precision=None, les=False):
    size = (2 * math.pi, math.pi, 1.0) if les else (4 * math.pi, 2 * math.pi, 2.0)
    if les:
        dom = api.Domain(size, api.RoughWall(1e-4), api.FreeSlipBoundary())
        procs = api.incompressible_flow(1e-5, constant_forcing=1, sgs_model=api.StaticSmagorinskyModel())
    else:
        dom = api.Domain(size, api.SmoothWall(), api.SmoothWall())
        procs = api.incompressible_flow(1 / 180, constant_forcing=1)
    kw = {} if precision is None else dict(precision=precision)
    return api.Model(res, dom, procs, **kw)


def _forced(BLD, family, res, precision, les=False):
    old = os.environ.get("BLD_X_KERNEL")
    os.environ["BLD_X_KERNEL"] = family
    try:
        return _build(BLD, res, precision, les)
    finally:
        if old is None:
            del os.environ["BLD_X_KERNEL"]
        else:
            os.environ["BLD_X_KERNEL"] = old


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


# (resolution, precision, tolerance): P1 = 96 (radix 3), 192 (6), 288 (9), 384 (12), 64 (2), 128 (4), 256 (8)
CASES = [
    ((192, 8, 5), "fp64", 1e-12),       # radix 9 in FP64: block kernels only (the warp-per-row one is FP32 there)
    ((64, 12, 6), "fp64", 1e-12),
    ((128, 10, 5), "fp64", 1e-12),
    ((43, 12, 6), "fp64", 1e-12),       # k1max = 21: P1 = 64, radix 2 (explicit 3k+1 rule)
    ((85, 10, 5), "fp64", 1e-12),       # k1max = 42: P1 = 128, radix 4
    ((64, 12, 6), "mixed", 1e-5),
    ((192, 8, 5), "mixed", 1e-5),
    ((256, 6, 4), "mixed", 1e-5),
    ((171, 6, 4), "mixed", 1e-5),       # k1max = 85: P1 = 256, radix 8
    ((341, 4, 4), "mixed", 1e-5),       # k1max = 170: P1 = 512, radix 16
    ((512, 4, 4), "mixed", 1e-5),       # k1max = 255: P1 = 768, radix 24
]


@pytest.mark.parametrize("res,precision,tol", CASES)
@pytest.mark.parametrize("family", ["warp", "block", "blockwarp", "pipe", "lines", "twopass"])
def test_advection_x_kernel_family(oracle, BLD, res, precision, tol, family):
    if family == "warp" and precision == "fp64" and res[0] == 192:
        pytest.skip("the warp-per-row kernel is compiled for radix <= 6 in FP64 (P1 = 288 is radix 9)")
    if family == "warp" and res[0] in (341, 512):
        pytest.skip("the warp-per-row kernel is compiled for radix <= 12 (P1 = 512, 768 are radix 16, 24)")
    om = _build(oracle, res)
    gm = _forced(BLD, family, res, precision)
    if family == "twopass":
        # two (double) or four (single precision) y rows per block
        if gm.info.adv_p2 % (2 if precision == "fp64" or gm.info.adv_p1 > 384 else 4) == 0:
            assert gm.kernels()["advection"]["x"].startswith("k_adv_x2<"), gm.kernels()
    elif family != "block":
        assert gm.info.adv_p1 % 32 == 0
    st = _state(om, seed=sum(res))
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (res, precision, family, gm.info.adv_p1, f, e)


@pytest.mark.parametrize("minb", ["3", "4"])
@pytest.mark.parametrize("res", [(171, 6, 4), (192, 8, 5), (256, 6, 4)])
def test_warp_x_kernel_register_caps(oracle, BLD, res, minb):
    """The warp-per-row x kernel compiled with a register cap (3 or 4 blocks of
    128 threads per SM; radices 8, 9, 12), forced, against the oracle (1e-5)."""
    saved = {k: os.environ.get(k) for k in ("BLD_X_KERNEL", "BLD_XW_MINB")}
    os.environ["BLD_X_KERNEL"] = "warp"
    os.environ["BLD_XW_MINB"] = minb
    try:
        gm = _build(BLD, res, "mixed")
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    xk = gm.kernels()["advection"]["x"]
    assert xk.startswith("k_adv_xwc<") and xk.endswith(", %s>" % minb), xk
    om = _build(oracle, res)
    st = _state(om, seed=sum(res) + int(minb))
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-5, (res, minb, f, e)


@pytest.mark.parametrize("family", ["warp", "blockwarp", "pipe", "twopass"])
def test_warp_kernel_les_mixed_trajectory(oracle, BLD, family):
    """The warp advection kernels inside a full LES step sequence (mixed form)."""
    res = (64, 64, 16)
    om = _build(oracle, res, les=True)
    gm = _forced(BLD, family, res, "mixed", les=True)
    st = _state(om, seed=5)
    for f in st:
        st[f] *= 5.0
    gm.set_state(st)
    for f in om.fields:
        om.state[f][...] = st[f]
    gm.evolve(10 * 1e-4, 1e-4)
    om.evolve(10 * 1e-4, 1e-4)
    got = gm.state
    for f in om.fields:
        e = rel_l2(got[f], om.state[f])
        assert e < 1e-5, (f, e)


def test_twopass_x_dns_trajectory(oracle, BLD):
    """20 SSP-RK33 steps of a DNS with the two-pass x kernel (P1 = 96) in the
    plain form, against the oracle at the trajectory tolerance (1e-9)."""
    res = (64, 32, 12)
    om = _build(oracle, res)
    gm = _forced(BLD, "twopass", res, "fp64")
    assert gm.kernels()["advection"]["x"].startswith("k_adv_x2<"), gm.kernels()
    st = _state(om, seed=12)
    for f in st:
        st[f] *= 20.0
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    om.evolve(20 * 1e-4, 1e-4)
    gm.evolve(20 * 1e-4, 1e-4)
    got = gm.state
    for f in om.fields:
        e = rel_l2(got[f], om.state[f])
        assert e < 1e-9, (f, e)


def _forced_y(BLD, family, res, precision, les):
    old = os.environ.get("BLD_Y_KERNEL")
    os.environ["BLD_Y_KERNEL"] = family
    try:
        return _build(BLD, res, precision, les)
    finally:
        if old is None:
            del os.environ["BLD_Y_KERNEL"]
        else:
            os.environ["BLD_Y_KERNEL"] = old


# y-pass sizes P2 = 96 (3), 288 (9), 384 (12), 64 (2), 192 (6), 128 (4), 256 (8), 512 (16), 768 (24)
Y_CASES = [
    ((16, 64, 6), "fp64", False, 1e-12),
    ((16, 192, 5), "fp64", False, 1e-12),
    ((16, 192, 5), "mixed", False, 1e-5),
    ((12, 256, 4), "mixed", False, 1e-5),
    ((32, 64, 8), "fp64", True, 1e-12),
    ((16, 128, 6), "mixed", True, 1e-5),
    ((12, 256, 4), "fp64", True, 1e-12),
    ((8, 512, 4), "fp64", True, 1e-12),
    ((8, 512, 4), "mixed", False, 1e-5),    # advection P2 = 768: radix 24 (single precision)
]


def _y3_fits(p2, n2, precision):
    """The TMA inverse y kernel runs where a TMA box holds whole k2 columns
    (K2 <= 256) and its staged tiles fit a block's shared memory."""
    k2 = 2 * ((n2 - 1) // 2) + 1
    al = lambda b: (b + 127) // 128 * 128
    cs = 8 if precision == "mixed" else 16
    return k2 <= 256 and 128 + al(p2 * cs) + al(p2 * 8 * cs) + 6 * al(k2 * 8 * 16) <= 227 * 1024


# P2 with a two-pass y kernel: both precisions, and single precision only
Y2_SIZES = {64, 96, 128, 144, 192, 256, 288}
Y2_SIZES_FP32 = {384, 512, 768}


@pytest.mark.parametrize("res,precision,les,tol", Y_CASES)
@pytest.mark.parametrize("family", ["warp", "block", "twopass", "twopass8", "twopass2", "tma"])
def test_y_kernel_family(oracle, BLD, res, precision, les, tol, family):
    om = _build(oracle, res, les=les)
    gm = _forced_y(BLD, family, res, precision, les)
    if family in ("twopass", "twopass8", "twopass2", "tma"):   # the forced family is the one that runs where it is compiled
        inv = "k_inv_y3<" if family == "tma" else "k_inv_y2<"
        for space in gm.kernels().values():
            if not isinstance(space, dict):
                continue
            p2 = space["P"][1]
            if family == "tma" and not _y3_fits(p2, res[1], precision):
                continue
            if p2 in Y2_SIZES or (precision == "mixed" and p2 in Y2_SIZES_FP32):
                assert space["inv_y"].startswith(inv) and space["fwd_y"].startswith("k_fwd_y2<"), space
                assert (family == "twopass8") == space["fwd_y"].endswith(", 8 lines>"), space
                assert (family == "twopass2" and precision == "mixed") == space["fwd_y"].endswith(", 2 outputs>"), space
    st = _state(om, seed=sum(res) + 1)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (res, precision, family, f, e)


@pytest.mark.parametrize("family", ["twopass", "twopass8"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_twopass_y_trajectory(oracle, BLD, precision, tol, family):
    """20 SSP-RK33 steps of an LES with both spaces on the two-pass y kernels
    (advection P2 = 96, SGS P2 = 64): the forward pass forms the fused stage
    values and the chained Euler stages, checked against the oracle."""
    res = (32, 64, 8)
    om = _build(oracle, res, les=True)
    gm = _forced_y(BLD, family, res, precision, True)
    for space in gm.kernels().values():
        if isinstance(space, dict):
            assert space["fwd_y"].startswith("k_fwd_y2<"), space
    st = _state(om, seed=77)
    om.apply_projections(st)
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    om.evolve(20 * 1e-4, 1e-4)
    gm.evolve(20 * 1e-4, 1e-4)
    got = gm.state
    for f in om.fields:
        e = rel_l2(got[f], om.state[f])
        assert e < tol, (precision, f, e)


# LES: the SGS x kernel (block Stockham or warp line transforms) with the advection
# kernel of the same family; P1 (SGS, advection) = (64, 96), (128, 192), (256, 384), (512, 768)
SGS_CASES = [
    ((64, 12, 6), "fp64", 1e-12),
    ((128, 8, 5), "mixed", 1e-5),
    ((256, 6, 4), "fp64", 1e-12),
    ((512, 4, 4), "mixed", 1e-5),
]


@pytest.mark.parametrize("res,precision,tol", SGS_CASES)
@pytest.mark.parametrize("family", ["block", "lines", "twopass"])
def test_sgs_x_kernel_family(oracle, BLD, res, precision, tol, family):
    om = _build(oracle, res, les=True)
    if family == "twopass":   # the SGS x pass on two-pass line transforms (BLD_SGS_X_KERNEL)
        old = os.environ.get("BLD_SGS_X_KERNEL")
        os.environ["BLD_SGS_X_KERNEL"] = "twopass"
        try:
            gm = _build(BLD, res, precision, les=True)
        finally:
            if old is None:
                del os.environ["BLD_SGS_X_KERNEL"]
            else:
                os.environ["BLD_SGS_X_KERNEL"] = old
        p1 = gm.info.sgs_p1
        if p1 <= 288 or precision == "mixed":
            xk = gm.kernels()["sgs"]["x"]
            assert xk.endswith(", 0, %d>" % p1) or xk.endswith(", 0, %d, 2>" % p1), gm.kernels()
    else:
        gm = _forced(BLD, family, res, precision, les=True)
    st = _state(om, seed=sum(res) + 2)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (res, precision, family, f, e)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_sgs_twopass_les_trajectory(oracle, BLD, precision, tol):
    """20 SSP-RK33 steps of an LES (64^2 x 16: SGS P1 = 64) with the SGS x pass
    on two-pass line transforms, against the oracle."""
    res = (64, 64, 16)
    om = _build(oracle, res, les=True)
    old = os.environ.get("BLD_SGS_X_KERNEL")
    os.environ["BLD_SGS_X_KERNEL"] = "twopass"
    try:
        gm = _build(BLD, res, precision, les=True)
    finally:
        if old is None:
            del os.environ["BLD_SGS_X_KERNEL"]
        else:
            os.environ["BLD_SGS_X_KERNEL"] = old
    assert gm.kernels()["sgs"]["x"].endswith(", 0, 64>"), gm.kernels()
    st = _state(om, seed=21)
    for f in st:
        st[f] *= 5.0
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    gm.evolve(20 * 1e-4, 1e-4)
    om.evolve(20 * 1e-4, 1e-4)
    got = gm.state
    for f in om.fields:
        e = rel_l2(got[f], om.state[f])
        assert e < tol, (precision, f, e)


@pytest.mark.parametrize("variant", ["0", "1", "2", "3"])
@pytest.mark.parametrize("res", [(16, 12, 7), (24, 20, 40), (16, 16, 200)])
def test_projection_variants(oracle, BLD, variant, res):
    """Column kernel (0), z-segmented kernels (1, 2) and the shared-tile one (3, n3 <= 128),
    each forced, against the oracle's projection (1e-12)."""
    if variant == "3" and res[2] > 128:
        pytest.skip("the tile variant is for n3 <= 128")
    old = os.environ.get("BLD_PROJ_VARIANT")
    os.environ["BLD_PROJ_VARIANT"] = variant
    try:
        gm = _build(BLD, res, "fp64")
    finally:
        if old is None:
            del os.environ["BLD_PROJ_VARIANT"]
        else:
            os.environ["BLD_PROJ_VARIANT"] = old
    om = _build(oracle, res)
    rng = np.random.default_rng(int(variant) + sum(res))
    st = {f: rng.standard_normal(om.state[f].shape) + 1j * rng.standard_normal(om.state[f].shape)
          for f in om.fields}
    ref = om.apply_projections({f: v.copy() for f, v in st.items()})
    got = gm.apply_projections({f: v.copy() for f, v in st.items()})
    for f in om.fields:
        assert rel_l2(got[f], ref[f]) < 1e-12, (variant, res, f)
    # and inside time steps (stage updates of SSPRK33)
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    gm.evolve(3 * 1e-3, 1e-3)
    om.evolve(3 * 1e-3, 1e-3)
    for f in om.fields:
        assert rel_l2(gm.state[f], om.state[f]) < 1e-10, (variant, res, f)


def test_bounded_wait_timeout_exit(oracle, BLD):
    """The TMA-staged x kernel's bounded wait taken to its timeout exit: with the
    device's wait limit set to 0 every block gives up at its first wait, lets the
    copies it issued land, sets the member's timeout flag and returns; the call
    reports BLD_ERR_TIMEOUT.  With the limit restored the same handle computes the
    rates exactly again (the context stays usable)."""
    from BoundaryLayerDynamics import _capi
    res = (64, 64, 6)
    gm = _forced(BLD, "twopass", res, "fp64")
    assert gm.kernels()["advection"]["x"].startswith("k_adv_x2<"), gm.kernels()
    om = _build(oracle, res)
    st = _state(om, seed=11)
    ref = om.compute_rates(st)
    lib = _capi.load()
    _capi.check(lib.bld_set_wait_limit(0, 0))
    try:
        with pytest.raises(_capi.BldError) as err:
            gm.compute_rates(st)
        assert err.value.status == _capi.BLD_ERR_TIMEOUT, err.value
    finally:
        _capi.check(lib.bld_set_wait_limit(0, -1))
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-12, (f, e)


@pytest.mark.parametrize("variant,name", [("0", ""), ("2", ", wide")])
@pytest.mark.parametrize("res", [(192, 8, 5), (64, 12, 6), (128, 10, 5), (85, 10, 5)])
def test_twopass_x_variants_fp64(oracle, BLD, res, variant, name):
    """The double-precision variants of the two-pass x kernel (as compiled, and
    with 1.5x the threads), forced, against the oracle at 1e-12."""
    saved = {k: os.environ.get(k) for k in ("BLD_X_KERNEL", "BLD_X2_VARIANT")}
    os.environ["BLD_X_KERNEL"] = "twopass"
    os.environ["BLD_X2_VARIANT"] = variant
    try:
        gm = _build(BLD, res, "fp64")
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    xk = gm.kernels()["advection"]["x"]
    assert xk.startswith("k_adv_x2<double") and xk.endswith(name + ">"), xk
    om = _build(oracle, res)
    st = _state(om, seed=sum(res) + int(variant))
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-12, (res, variant, f, e)


def _project_pipe_smem(n3, ln):
    """Dynamic shared memory of k_project_pipe: slack and barriers, two stages of
    three component tiles (n3 ln values rounded up to 8) and gamma."""
    stride = (n3 * ln + 7) // 8 * 8
    stage = (3 * stride * 16 + n3 * ln * 8 + 127) // 128 * 128
    return 256 + 2 * stage


@pytest.mark.parametrize("pipe", ["0", "1"])
@pytest.mark.parametrize("tile", ["4", "8", "16"])
@pytest.mark.parametrize("res,flux", [((16, 12, 7), False), ((24, 20, 40), True), ((16, 16, 200), False),
                                      ((64, 64, 96), True), ((17, 12, 9), False)])
def test_projection_tile(oracle, BLD, tile, pipe, res, flux):
    """k_project_tile (each block's columns brought into shared memory by TMA
    tensor copies, 4, 8 or 16 columns per block), and its persistent two-stage
    form k_project_pipe where two stages fit in 200 KB, forced for the
    projections of stored stage values: apply_projections and 10 chained
    SSP-RK33 steps against the oracle, with and without ConstantMean.  An odd
    number of modes per layer (17 x 12: F = 9 x 11) keeps the z-segmented
    kernel."""
    saved = {k: os.environ.get(k) for k in ("BLD_PROJ_TILE", "BLD_PROJ_PIPE")}
    os.environ["BLD_PROJ_TILE"] = tile
    os.environ["BLD_PROJ_PIPE"] = pipe

    def build(api):
        dom = api.Domain((4 * math.pi, 2 * math.pi, 2.0), api.SmoothWall(), api.SmoothWall())
        procs = (api.incompressible_flow(1 / 180, constant_flux=(1.0, 0.3)) if flux
                 else api.incompressible_flow(1 / 180, constant_forcing=1))
        return api.Model(res, dom, procs)
    try:
        gm = build(BLD)
    finally:
        for k, v in saved.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    om = build(oracle)
    F = om.state["vel1"].shape[1] * om.state["vel1"].shape[2]
    stored = gm.kernels().get("projection_stored", "")
    if F % 2 == 0:
        persistent = pipe == "1" and _project_pipe_smem(res[2], int(tile)) <= 200 * 1024
        name = "k_project_pipe" if persistent else "k_project_tile"
        assert stored == "%s<%d, %s>" % (name, 8 if res[2] <= 128 else 16, tile), gm.kernels()
    else:
        assert stored == "", gm.kernels()
    rng = np.random.default_rng(int(tile) + sum(res))
    st = {f: rng.standard_normal(om.state[f].shape) + 1j * rng.standard_normal(om.state[f].shape)
          for f in om.fields}
    ref = om.apply_projections({f: v.copy() for f, v in st.items()})
    got = gm.apply_projections({f: v.copy() for f, v in st.items()})
    for f in om.fields:
        assert rel_l2(got[f], ref[f]) < 1e-12, (tile, res, f)
    st = _state(om, seed=int(tile) + 7)
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    gm.evolve(10 * 1e-4, 1e-4)
    om.evolve(10 * 1e-4, 1e-4)
    for f in om.fields:
        e = rel_l2(gm.state[f], om.state[f])
        assert e < 1e-10, (tile, res, f, e)


@pytest.mark.parametrize("res", [(256, 6, 4), (512, 4, 4)])
def test_sgs_twopass_capped(oracle, BLD, res):
    """The single-precision two-pass SGS x kernel compiled for two blocks of 256
    threads per SM (registers capped at 128), forced, against the oracle (1e-5)."""
    om = _build(oracle, res, les=True)
    old = os.environ.get("BLD_SGS_X_KERNEL")
    os.environ["BLD_SGS_X_KERNEL"] = "twopass_capped"
    try:
        gm = _build(BLD, res, "mixed", les=True)
    finally:
        if old is None:
            del os.environ["BLD_SGS_X_KERNEL"]
        else:
            os.environ["BLD_SGS_X_KERNEL"] = old
    assert gm.kernels()["sgs"]["x"].endswith(", 0, %d, 2>" % gm.info.sgs_p1), gm.kernels()
    st = _state(om, seed=sum(res) + 5)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-5, (res, f, e)


@pytest.mark.parametrize("res,precision,tol,sgs_sizes", [((64, 12, 6), "fp64", 1e-12, None),
                                                         ((128, 8, 5), "mixed", 1e-5, None),
                                                         ((512, 4, 4), "mixed", 1e-5, None),
                                                         ((58, 12, 5), "mixed", 1e-5, (96, 96))])
def test_sgs_twopass_staged(oracle, BLD, res, precision, tol, sgs_sizes):
    """The two-pass SGS x kernel with its input rows staged in shared memory by 1-d
    TMA bulk copies one layer ahead (forced), against the oracle.  The last case
    runs the Smagorinsky model at an explicit 96 x 96 grid for 58 x 12 modes:
    K1 = 29 single-precision values per row, so a block takes an even number of
    rows to fill whole 16-byte units."""
    def build(api, prec=None):
        if sgs_sizes is None:
            return _build(api, res, prec, les=True)
        dom = api.Domain((2 * math.pi, math.pi, 1.0), api.RoughWall(1e-4), api.FreeSlipBoundary())
        procs = api.incompressible_flow(1e-5, constant_forcing=1,
                                        sgs_model=api.StaticSmagorinskyModel(dealiasing=sgs_sizes))
        kw = {} if prec is None else dict(precision=prec)
        return api.Model(res, dom, procs, **kw)
    om = build(oracle)
    old = os.environ.get("BLD_SGS_X_KERNEL")
    os.environ["BLD_SGS_X_KERNEL"] = "twopass_staged"
    try:
        gm = build(BLD, precision)
    finally:
        if old is None:
            del os.environ["BLD_SGS_X_KERNEL"]
        else:
            os.environ["BLD_SGS_X_KERNEL"] = old
    xk = gm.kernels()["sgs"]["x"]
    assert xk.startswith("k_sgs_x<") and ", 0, %d" % gm.info.sgs_p1 in xk, gm.kernels()
    st = _state(om, seed=sum(res) + 9)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (res, precision, f, e)


@pytest.mark.parametrize("res,precision,tol", [((64, 12, 6), "fp64", 1e-12), ((64, 12, 6), "mixed", 1e-5),
                                               ((96, 8, 5), "mixed", 1e-5), ((128, 8, 5), "mixed", 1e-5),
                                               ((128, 8, 5), "fp64", 1e-12), ((256, 6, 4), "fp64", 1e-12),
                                               ((512, 4, 4), "mixed", 1e-5)])
def test_sgs_rows_kernel(oracle, BLD, res, precision, tol):
    """k_sgs_x2 (rows staged by 1-d TMA bulk copies, two-pass line transforms, one
    thread per pass-1 task) forced with BLD_SGS_X_KERNEL=rows, against the oracle."""
    om = _build(oracle, res, les=True)
    old = os.environ.get("BLD_SGS_X_KERNEL")
    os.environ["BLD_SGS_X_KERNEL"] = "rows"
    try:
        gm = _build(BLD, res, precision, les=True)
    finally:
        if old is None:
            del os.environ["BLD_SGS_X_KERNEL"]
        else:
            os.environ["BLD_SGS_X_KERNEL"] = old
    assert gm.kernels()["sgs"]["x"].startswith("k_sgs_x2<"), gm.kernels()
    st = _state(om, seed=sum(res) + 13)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < tol, (res, precision, f, e)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_sgs_rows_kernel_trajectory(oracle, BLD, precision, tol):
    """20 SSP-RK33 steps of a 64 x 64 x 8 LES with k_sgs_x2 forced (z chunks,
    the carried values and the wall model across layers), against the oracle."""
    res = (64, 64, 8)
    om = _build(oracle, res, les=True)
    old = os.environ.get("BLD_SGS_X_KERNEL")
    os.environ["BLD_SGS_X_KERNEL"] = "rows"
    try:
        gm = _build(BLD, res, precision, les=True)
    finally:
        if old is None:
            del os.environ["BLD_SGS_X_KERNEL"]
        else:
            os.environ["BLD_SGS_X_KERNEL"] = old
    assert gm.kernels()["sgs"]["x"].startswith("k_sgs_x2<"), gm.kernels()
    st = _state(om, seed=21)
    gm.set_state(st)
    om.state.update({f: v.copy() for f, v in st.items()})
    gm.evolve(20 * 1e-4, 1e-4)
    om.evolve(20 * 1e-4, 1e-4)
    for f in om.fields:
        e = rel_l2(gm.state[f], om.state[f])
        assert e < tol, (precision, f, e)


def _with_env(env, fn):
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return fn()
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("kind", ["projection_tile", "projection_pipe", "sgs_rows", "sgs_staged"])
def test_bounded_wait_timeout_exit_other_kernels(oracle, BLD, kind):
    """The timeout exit of the other kernels that wait for their own TMA copies
    (the tile projection and its persistent form, the SGS x kernel with staged row groups, the two-pass
    SGS x kernel with staged rows), each forced, with the device's wait limit at
    0: the call reports BLD_ERR_TIMEOUT; with the limit restored the same handle
    gives the oracle's result again."""
    from BoundaryLayerDynamics import _capi
    if kind.startswith("projection"):
        res, les = (64, 64, 6), False
        env = {"BLD_PROJ_TILE": "8", "BLD_PROJ_PIPE": "1" if kind == "projection_pipe" else "0"}
    elif kind == "sgs_rows":
        res, les, env = (64, 12, 6), True, {"BLD_SGS_X_KERNEL": "rows"}
    else:
        res, les, env = (64, 12, 6), True, {"BLD_SGS_X_KERNEL": "twopass_staged"}
    gm = _with_env(env, lambda: _build(BLD, res, "fp64", les=les))
    om = _build(oracle, res, les=les)
    if kind.startswith("projection"):
        name = "k_project_pipe<" if kind == "projection_pipe" else "k_project_tile<"
        assert gm.kernels()["projection_stored"].startswith(name), gm.kernels()
        rng = np.random.default_rng(5)
        st = {f: rng.standard_normal(om.state[f].shape) + 1j * rng.standard_normal(om.state[f].shape)
              for f in om.fields}
        call = lambda g: g.apply_projections({f: v.copy() for f, v in st.items()})
    else:
        st = _state(om, seed=17)
        call = lambda g: g.compute_rates(st)
    ref = call(om)
    lib = _capi.load()
    _capi.check(lib.bld_set_wait_limit(0, 0))
    try:
        with pytest.raises(_capi.BldError) as err:
            call(gm)
        assert err.value.status == _capi.BLD_ERR_TIMEOUT, err.value
    finally:
        _capi.check(lib.bld_set_wait_limit(0, -1))
    got = call(gm)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-12, (kind, f, e)


@pytest.mark.parametrize("res", [(192, 8, 5), (64, 12, 6), (256, 6, 4)])
def test_twopass_x_two_rows_mixed(oracle, BLD, res):
    """The single-precision two-pass x kernel with two rows per block (four blocks
    of four warps per SM instead of two of seven), forced, against the oracle at
    the mixed form's 1e-5."""
    gm = _with_env({"BLD_X_KERNEL": "twopass", "BLD_X2_VARIANT": "3"}, lambda: _build(BLD, res, "mixed"))
    xk = gm.kernels()["advection"]["x"]
    assert xk.startswith("k_adv_x2<float") and xk.endswith(", 2 rows>"), xk
    om = _build(oracle, res)
    st = _state(om, seed=sum(res) + 31)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-5, (res, f, e)


@pytest.mark.parametrize("res", [(64, 12, 6), (128, 8, 5), (96, 8, 5)])
def test_sgs_rows_kernel_two_rows_mixed(oracle, BLD, res):
    """k_sgs_x2 with two rows per block in single precision (smaller blocks, more
    per SM), forced, against the oracle at the mixed form's 1e-5."""
    gm = _with_env({"BLD_SGS_X_KERNEL": "rows", "BLD_SGS_X2_VARIANT": "1"},
                   lambda: _build(BLD, res, "mixed", les=True))
    xk = gm.kernels()["sgs"]["x"]
    assert xk.startswith("k_sgs_x2<float") and xk.endswith(", 2 rows>"), xk
    om = _build(oracle, res, les=True)
    st = _state(om, seed=sum(res) + 41)
    ref = om.compute_rates(st)
    got = gm.compute_rates(st)
    for f in om.fields:
        e = rel_l2(got[f], ref[f])
        assert e < 1e-5, (res, f, e)
