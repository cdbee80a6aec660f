"""Uneven ensembles: independent members of several grid sizes advanced together.

The reference runs one ``Model`` per process.  Here members of one size share a
handle (``Model(..., members=B)``): every kernel of the right-hand side and of
the projection runs once per stage for all B members, with per-member Cs,
roughness length and forcing tables.  The size classes of an uneven ensemble
are separate handles on one device, and ``Ensemble.step`` advances all of them
with ONE CUDA-graph launch per time step: a parent graph whose independent
child graphs are the classes' step graphs (``bld_ensemble_step``), so the
classes overlap on the device and the host issues a single launch per step.
"""

import ctypes as C
import sys

from . import _capi, _METHODS, SSPRK33
from . import workloads


class Ensemble:
    """Size classes (``Model`` handles with ``members`` slots each) stepped as one graph."""

    def __init__(self, models):
        self.models = list(models)
        if not self.models:
            raise ValueError("an ensemble needs at least one size class")

    @classmethod
    def from_groups(cls, groups, precision="mixed", device=0):
        """``groups``: dicts with ``spec`` (a workload spec), ``z0`` and ``cs`` (one value per member)."""
        api = sys.modules[__package__]
        models = []
        for g in groups:
            models.append(workloads.build(g["spec"], api, precision=precision, members=len(g["z0"]),
                                          device=device, member_cs=g["cs"], member_z0=g["z0"]))
        return cls(models)

    @property
    def points(self):
        """Grid points advanced per step, summed over all members (N1*N2*N3 each)."""
        return sum(m.members * m.resolution[0] * m.resolution[1] * m.resolution[2] for m in self.models)

    @property
    def members(self):
        return sum(m.members for m in self.models)

    def prepare(self):
        for m in self.models:
            m.prepare()

    def step(self, nsteps, dt, method=SSPRK33):
        """``nsteps`` steps of every member: one graph launch per step; checks divergence."""
        step_models(self.models, nsteps, dt, method)

    def initialize(self, groups, seed=0):
        """Seeded log-law-plus-noise initial fields (each member with its own roughness length)."""
        k = 0
        for m, g in zip(self.models, groups):
            for i in range(m.members):
                spec = dict(g["spec"])
                spec["lower"] = ("rough", float(g["z0"][i]))
                u, v, w = workloads.initial_fields(spec, seed=seed + k)
                m.set_field("vel1", u, member=i)
                m.set_field("vel2", v, member=i)
                m.set_field("vel3", w, member=i)
                k += 1


def step_models(models, nsteps, dt, method=SSPRK33):
    """Advances the handles of ``models`` (one device) by ``nsteps`` steps, one parent-graph
    launch per step (``bld_ensemble_step``); raises DivergenceError if any member diverged."""
    handles = (C.c_void_p * len(models))(*[m._h.value for m in models])
    _capi.check(_capi.load().bld_ensemble_step(handles, len(models), int(nsteps), float(dt), _METHODS[method]))
