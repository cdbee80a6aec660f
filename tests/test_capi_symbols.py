"""CPU checks of the C ABI: the library loads, exports every declared symbol and
rejects work cleanly when no device is present."""

import ctypes
import importlib.util
import os
import re

import pytest

from conftest import PKG_DIR, REPO

HEADER = os.path.join(REPO, "include", "bld.h")


def _build():
    spec = importlib.util.spec_from_file_location("bld_build", os.path.join(PKG_DIR, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int32_t|void|const char\*)\s+(bld_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    path = _build()
    return ctypes.CDLL(path)


def test_header_declares_the_abi():
    names = declared_functions()
    for n in ("bld_create", "bld_destroy", "bld_compute_rates", "bld_apply_projections", "bld_evolve", "bld_step"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from BoundaryLayerDynamics import _capi
    assert set(declared_functions()) == set(_capi.SIGNATURES)


def test_status_strings(lib):
    from BoundaryLayerDynamics import _capi
    L = _capi.load()
    assert L.bld_abi_version() == 1
    assert L.bld_status_string(_capi.BLD_ERR_DIVERGED) == b"The simulation has diverged."


def test_create_validates_before_touching_a_device():
    """Invalid configurations are rejected with the reference's messages (no GPU needed)."""
    import math
    import BoundaryLayerDynamics as BLD
    from BoundaryLayerDynamics import _capi
    with pytest.raises(ValueError, match="at least 3 vertical layers"):
        BLD.Model((8, 8, 2), BLD.Domain((1, 1, 1), BLD.SmoothWall(), BLD.SmoothWall()), [BLD.Pressure()])
    dom = BLD.Domain((1, 1, 1), BLD.CustomBoundary(vel1="dirichlet", vel2="dirichlet", vel3=("dirichlet", 1.0)),
                     BLD.CustomBoundary(vel1="dirichlet", vel2="dirichlet", vel3=("dirichlet", 2.0)))
    with pytest.raises(_capi.BldError, match="mean flow must be equal"):
        BLD.Model((8, 8, 4), dom, [BLD.Pressure()])
    dom = BLD.Domain((2 * math.pi, math.pi, 1), BLD.SmoothWall(), BLD.FreeSlipBoundary())
    with pytest.raises(_capi.BldError, match="rough-wall and free-slip"):
        BLD.Model((8, 8, 4), dom, [BLD.StaticSmagorinskyModel()])


def test_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import BoundaryLayerDynamics as BLD
    from BoundaryLayerDynamics import _capi
    with pytest.raises(_capi.BldError) as e:
        BLD.closedchannelflow(180, (8, 8, 4))
    assert e.value.status == _capi.BLD_ERR_NO_DEVICE
