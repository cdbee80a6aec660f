"""Writes the golden fixtures of this directory from the oracle.

The reference ships no golden vectors and cannot run here (no Julia), so the
oracle, pinned by the reference's own known-answer tests, is the source.  The
fixtures freeze its outputs on seeded inputs: a later change of the oracle that
alters results is caught by tests/test_golden.py on the CPU, and the engine is
compared with the same files on the GPU.

    python tests/golden/make_golden.py
"""

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "oracle"), os.path.join(REPO, "boundarylayerdynamics.jl_b200")]


def cases(api):
    """(name, model, kind) for each fixture; ``api`` is the oracle or the engine binding."""
    dns = api.Model((12, 12, 6), api.Domain((4 * math.pi, 2 * math.pi, 2.0), api.SmoothWall(), api.SmoothWall()),
                    api.incompressible_flow(1 / 180, constant_forcing=1))
    les = api.Model((12, 12, 6), api.Domain((2 * math.pi, math.pi, 1.0), api.RoughWall(1e-4), api.FreeSlipBoundary()),
                    api.incompressible_flow(1e-5, constant_forcing=1, sgs_model=api.StaticSmagorinskyModel()))
    return [("dns_12x12x6", dns), ("les_12x12x6", les)]


def seeded_state(model, seed):
    rng = np.random.default_rng(seed)
    st = {}
    for f in ("vel1", "vel2", "vel3"):
        shape = model.state[f].shape
        k1 = np.arange(shape[2])[None, None, :]
        k2 = np.abs(np.concatenate([np.arange(shape[1] // 2 + 1), -np.arange(shape[1] // 2, 0, -1)]))[None, :, None]
        st[f] = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / (1.0 + k1 ** 2 + k2 ** 2)
        st[f][:, 0, 0] = st[f][:, 0, 0].real
    return st


def main():
    import bld_oracle as O
    for i, (name, om) in enumerate(cases(O)):
        st = seeded_state(om, 100 + i)
        rates = om.compute_rates({f: v.copy() for f, v in st.items()})
        proj = om.apply_projections({f: v.copy() for f, v in st.items()})
        for f in om.fields:
            om.state[f][...] = proj[f]
        om.evolve(10 * 2.0 ** -10, 2.0 ** -10)
        out = {}
        for f in om.fields:
            out[f"in_{f}"] = st[f]
            out[f"rates_{f}"] = rates[f]
            out[f"proj_{f}"] = proj[f]
            out[f"traj_{f}"] = om.state[f]
            out[f"phys_{f}"] = om.get_field(f, centered=True)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
