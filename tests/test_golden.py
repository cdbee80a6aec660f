"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py).

CPU: the oracle still reproduces its frozen outputs (rates, projection, a
10-step SSP-RK33 trajectory, centered physical fields) to round-off, so a change
of the oracle cannot silently move the parity target.  GPU: the engine matches
the same files at the parity bars (1e-12 for rates and projections, 1e-9 for
the trajectory and the physical fields).
"""

import os
import sys

import numpy as np
import pytest

from conftest import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

FIELDS = ("vel1", "vel2", "vel3")
DT = 2.0 ** -10


def _fixture(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


@pytest.mark.parametrize("idx", [0, 1])
def test_oracle_reproduces_golden(oracle, idx):
    name, om = make_golden.cases(oracle)[idx]
    fx = _fixture(name)
    st = {f: fx[f"in_{f}"] for f in FIELDS}
    rates = om.compute_rates({f: v.copy() for f, v in st.items()})
    proj = om.apply_projections({f: v.copy() for f, v in st.items()})
    for f in FIELDS:
        assert rel_l2(rates[f], fx[f"rates_{f}"]) < 1e-13, (name, f)
        assert rel_l2(proj[f], fx[f"proj_{f}"]) < 1e-13, (name, f)
        om.state[f][...] = proj[f]
    om.evolve(10 * DT, DT)
    for f in FIELDS:
        assert rel_l2(om.state[f], fx[f"traj_{f}"]) < 1e-12, (name, f)
        assert rel_l2(om.get_field(f, centered=True), fx[f"phys_{f}"]) < 1e-12, (name, f)


@pytest.mark.gpu
@pytest.mark.parametrize("idx", [0, 1])
def test_engine_matches_golden(idx):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import BoundaryLayerDynamics as BLD
    name, gm = make_golden.cases(BLD)[idx]
    fx = _fixture(name)
    st = {f: fx[f"in_{f}"] for f in FIELDS}
    rates = gm.compute_rates(st)
    proj = gm.apply_projections({f: v.copy() for f, v in st.items()})
    for f in FIELDS:
        assert rel_l2(rates[f], fx[f"rates_{f}"]) < 1e-12, (name, f)
        assert rel_l2(proj[f], fx[f"proj_{f}"]) < 1e-12, (name, f)
    gm.set_state(proj)
    gm.evolve(10 * DT, DT)
    state = gm.state
    for f in FIELDS:
        assert rel_l2(state[f], fx[f"traj_{f}"]) < 1e-9, (name, f)
        assert rel_l2(gm.get_field(f, centered=True), fx[f"phys_{f}"]) < 1e-9, (name, f)
