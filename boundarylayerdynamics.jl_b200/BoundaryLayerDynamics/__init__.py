"""Host-side mirror of BoundaryLayerDynamics.jl's public API over the B200 engine.

Names, arguments and errors follow the reference (src/BoundaryLayerDynamics.jl,
src/Domains.jl, src/processes/*.jl): ``Model(resolution, domain, processes)``,
``initialize(model, vel1=f)`` (``initialize!``), ``model["vel1"]``
(``getindex``), ``evolve(model, tspan, dt=..., method=SSPRK33)`` (``evolve!``),
``incompressible_flow``, ``closedchannelflow``, ``openchannelflow`` and the
process constructors.  All computation runs in the CUDA library
``lib/libbld.so`` through its C ABI (include/bld.h); this module only
evaluates the domain mapping and initial conditions on the host and moves
arrays.

Extensions beyond the reference: ``precision="mixed"`` (FP32 transforms,
advection and SGS; FP64 state, linear terms, pressure solve and mean-mode
sources) and ``members=B`` (B independent ensemble members of one size, with
optional per-member ``Cs``, roughness length and forcing).
"""

import ctypes as C
import math
from fractions import Fraction

import numpy as np

from . import _capi
from ._capi import DivergenceError, BldError

__all__ = [
    "Model", "Domain", "SmoothWall", "RoughWall", "FreeSlipBoundary", "CustomBoundary", "SinusoidalMapping",
    "MomentumAdvection", "MolecularDiffusion", "Pressure", "ConstantSource", "ConstantMean",
    "StaticSmagorinskyModel", "incompressible_flow", "closedchannelflow", "openchannelflow",
    "initialize", "evolve", "reset", "coordinates", "Euler", "AB2", "SSPRK22", "SSPRK33",
    "DivergenceError", "BldError",
]

Euler, AB2, SSPRK22, SSPRK33 = "Euler", "AB2", "SSPRK22", "SSPRK33"
_METHODS = {Euler: _capi.EULER, AB2: _capi.AB2, SSPRK22: _capi.SSPRK22, SSPRK33: _capi.SSPRK33}
FIELDS = ("vel1", "vel2", "vel3")


# ----------------------------------------------------------------- domain (src/Domains.jl)
class SmoothWall:
    """No-slip, no-penetration wall (src/Domains.jl:173-179)."""


class RoughWall:
    """Rough wall with roughness length z0 (src/Domains.jl:181-192)."""

    def __init__(self, roughness, von_karman_constant=0.4):
        self.roughness, self.von_karman_constant = float(roughness), float(von_karman_constant)


class FreeSlipBoundary:
    """No-penetration boundary with vanishing tangential gradients (src/Domains.jl:194-200)."""


class CustomBoundary:
    """Explicit BCs: ``CustomBoundary(vel1=("dirichlet", 1.0), vel3="dirichlet")`` (src/Domains.jl:202-220)."""

    def __init__(self, **behaviors):
        self.behaviors = behaviors


class SinusoidalMapping:
    """Vertical grid stretching (src/Domains.jl:72-130)."""

    def __init__(self, eta, variant="auto"):
        if not 0 < eta < 1:
            raise ValueError("SinusoidalMapping needs 0 < eta < 1")
        self.parameter, self.variant = float(eta), variant


def _hasboundarylayer(b):
    if isinstance(b, (RoughWall, SmoothWall)):
        return True
    if isinstance(b, FreeSlipBoundary):
        return False
    raise ValueError("Could not determine variant of SinusoidalMapping")


def _f(z):
    return float(z) if isinstance(z, Fraction) else z


class Domain:
    """``Domain(dims, lower_boundary, upper_boundary, mapping=None)`` (src/Domains.jl:30-47,97-135)."""

    def __init__(self, dims, lower_boundary, upper_boundary, mapping=None):
        self.hsize = (float(dims[0]), float(dims[1]))
        if len(dims) == 2:
            lo, hi = 0.0, 1.0
        elif isinstance(dims[2], (tuple, list)):
            lo, hi = float(dims[2][0]), float(dims[2][1])
        else:
            lo, hi = 0.0, float(dims[2])
        self.lower_boundary, self.upper_boundary = lower_boundary, upper_boundary
        if mapping is None:
            l3 = hi - lo
            self._vmap = lambda z: lo + _f(z) * l3
            self._dvmap = lambda z: hi - lo
        elif isinstance(mapping, SinusoidalMapping):
            eta, l, pi = mapping.parameter, hi - lo, math.pi
            v = mapping.variant
            if v == "auto":
                v = {(True, True): "symmetric", (True, False): "below", (False, True): "above"}.get(
                    (_hasboundarylayer(lower_boundary), _hasboundarylayer(upper_boundary)))
                if v is None:
                    raise ValueError("Could not determine variant of SinusoidalMapping")
            s = math.sin(eta * pi / 2)
            if v == "symmetric":
                self._vmap = lambda z: lo + l / 2 * (1 + math.sin(eta * _f(2 * z - 1) * pi / 2) / s)
                self._dvmap = lambda z: l * eta * pi / 2 / s * math.cos(eta * _f(2 * z - 1) * pi / 2)
            elif v == "below":
                self._vmap = lambda z: lo + l * (1 + math.sin(eta * _f(z - 1) * pi / 2) / s)
                self._dvmap = lambda z: l * eta * pi / 2 / s * math.cos(eta * _f(z - 1) * pi / 2)
            elif v == "above":
                self._vmap = lambda z: lo + l * (math.sin(eta * _f(z) * pi / 2) / s)
                self._dvmap = lambda z: l * eta * pi / 2 / s * math.cos(eta * _f(z) * pi / 2)
            else:
                raise ValueError("Unknown variant of SinusoidalMapping")
        else:
            self._vmap, self._dvmap = mapping

    def vmap(self, z):
        return float(self._vmap(z))

    def Dvmap(self, z):
        return float(self._dvmap(z))

    def extrema3(self):
        return self.vmap(Fraction(0)), self.vmap(Fraction(1))


def _bctype(boundary, field):
    """(kind, value) per src/boundary_conditions.jl:85-95,53-59."""
    if isinstance(boundary, CustomBoundary):
        b = boundary.behaviors[field]
        kind, val = (b, 0.0) if isinstance(b, str) else (b[0], float(b[1]))
    elif isinstance(boundary, (SmoothWall, RoughWall)):
        kind, val = "dirichlet", 0.0
    elif isinstance(boundary, FreeSlipBoundary):
        kind, val = ("dirichlet", 0.0) if field == "vel3" else ("neumann", 0.0)
    else:
        raise ValueError(f"unknown boundary {boundary!r}")
    if kind not in ("dirichlet", "neumann"):
        raise ValueError(f"unsupported boundary behaviour {kind!r} for {field}")
    return (_capi.BC_DIRICHLET if kind == "dirichlet" else _capi.BC_NEUMANN), val


# ------------------------------------------------------------ processes (src/processes/*.jl)
class MomentumAdvection:
    def __init__(self, dealiasing="quadratic"):
        self.dealiasing = dealiasing


class MolecularDiffusion:
    def __init__(self, field, diffusivity):
        self.field, self.diffusivity = field, float(diffusivity)


class Pressure:
    def __init__(self, batch_size=64):
        self.batch_size = batch_size


class ConstantSource:
    def __init__(self, field, strength=1):
        self.field, self.strength = field, float(strength)


class ConstantMean:
    def __init__(self, field, mean_value=1):
        self.field, self.mean_value = field, float(mean_value)


class StaticSmagorinskyModel:
    def __init__(self, dealiasing=None, Cs=0.1, wall_damping=True, wall_damping_exponent=2):
        self.dealiasing, self.Cs = dealiasing, float(Cs)
        self.wall_damping, self.wall_damping_exponent = wall_damping, wall_damping_exponent


def incompressible_flow(viscosity, sgs_model=None, constant_forcing=None, constant_flux=None):
    """src/BoundaryLayerDynamics.jl:116-132"""
    if constant_flux is not None and constant_forcing is not None:
        raise ValueError("Momentum source set up for both constant forcing and constant flux")
    if constant_flux is None and constant_forcing is None:
        constant_forcing = 1
    procs = [MomentumAdvection()] + [MolecularDiffusion(v, viscosity) for v in FIELDS] + [Pressure()]
    if constant_forcing is not None:
        vals = constant_forcing if isinstance(constant_forcing, (tuple, list)) else (constant_forcing,)
        procs += [ConstantSource(("vel1", "vel2")[i], f) for i, f in enumerate(vals)]
    else:
        vals = constant_flux if isinstance(constant_flux, (tuple, list)) else (constant_flux,)
        procs += [ConstantMean(("vel1", "vel2")[i], m) for i, m in enumerate(vals)]
    if sgs_model is not None:
        procs.append(sgs_model)
    return procs


def _flatten(ps):
    for p in ps:
        if isinstance(p, (list, tuple)):
            yield from _flatten(p)
        else:
            yield p


def _dealias(d):
    if d is None:
        return _capi.DEALIAS_NONE, 0, 0
    if d == "quadratic":
        return _capi.DEALIAS_QUADRATIC, 0, 0
    if isinstance(d, tuple):
        return _capi.DEALIAS_EXPLICIT, int(d[0]), int(d[1])
    raise ValueError(f"Unsupported dealiasing type: {d}")


def _resolution(r):
    if isinstance(r, int):
        return (r, r, r)
    if len(r) == 2:
        return (r[0], r[0], r[1])
    return tuple(int(x) for x in r)


# ----------------------------------------------------------------------------- Model
class Model:
    """``Model(resolution, domain, processes)`` (src/BoundaryLayerDynamics.jl:72-97) on a B200.

    The state lives on the device; ``model.state`` reads it back as a dict of
    complex arrays of shape (n3, 2*k2max+1, k1max+1) (the reference layout).
    """

    def __init__(self, resolution, domain, processes, precision="fp64", members=1, device=0,
                 member_cs=None, member_z0=None, member_forcing=None):
        self._lib = _capi.load()
        self.domain = domain
        self.resolution = _resolution(resolution)
        n1, n2, n3 = self.resolution
        if n3 < 3:
            raise ValueError("Due to boundary stencils, the grid needs at least 3 vertical layers")
        self.k1max, self.k2max, self.n3 = (n1 - 1) // 2, (n2 - 1) // 2, n3
        self.K1, self.K2 = self.k1max + 1, 2 * self.k2max + 1
        self.members = int(members)
        self.processes = list(_flatten(processes))
        cfg = _capi.BldConfig()
        cfg.n1, cfg.n2, cfg.n3, cfg.members = n1, n2, n3, self.members
        cfg.l1, cfg.l2 = domain.hsize
        cfg.x3_min, cfg.x3_max = domain.extrema3()
        zc = [Fraction(2 * i - 1, 2 * n3) for i in range(1, n3 + 1)]
        zi = [Fraction(i, n3) for i in range(n3 + 1)]
        self._tables = {
            "dx3_c": np.array([domain.Dvmap(float(z)) for z in zc]),
            "dx3_i": np.array([domain.Dvmap(float(z)) for z in zi]),
            "x3_c": np.array([domain.vmap(z) for z in zc]),
            "x3_i": np.array([domain.vmap(z) for z in zi[1:-1]]),
        }
        for k, v in self._tables.items():
            setattr(cfg, k, v.ctypes.data_as(C.POINTER(C.c_double)))
        fields = set()
        for f in FIELDS:
            for s, b in enumerate((domain.lower_boundary, domain.upper_boundary)):
                try:
                    kind, val = _bctype(b, f)
                except (KeyError, ValueError):
                    kind, val = _capi.BC_DIRICHLET, 0.0
                    self._bc_missing = True
                cfg.bc_kind[FIELDS.index(f)][s] = kind
                cfg.bc_value[FIELDS.index(f)][s] = val
        for s, b in enumerate((domain.lower_boundary, domain.upper_boundary)):
            if isinstance(b, RoughWall):
                cfg.wall_kind[s], cfg.wall_z0[s], cfg.wall_kappa[s] = _capi.WALL_ROUGH, b.roughness, b.von_karman_constant
            elif isinstance(b, FreeSlipBoundary):
                cfg.wall_kind[s] = _capi.WALL_FREESLIP
            else:
                cfg.wall_kind[s] = _capi.WALL_OTHER
        for p in self.processes:
            if isinstance(p, MomentumAdvection):
                cfg.advection = 1
                cfg.adv_dealias, cfg.adv_p1, cfg.adv_p2 = _dealias(p.dealiasing)
                fields.update(FIELDS)
            elif isinstance(p, MolecularDiffusion):
                i = FIELDS.index(p.field)
                cfg.diffusion[i], cfg.diffusivity[i] = 1, p.diffusivity
                fields.add(p.field)
            elif isinstance(p, Pressure):
                cfg.pressure = 1
                fields.update(FIELDS)
            elif isinstance(p, ConstantSource):
                i = FIELDS.index(p.field)
                cfg.source[i], cfg.source_strength[i] = 1, p.strength
                fields.add(p.field)
            elif isinstance(p, ConstantMean):
                i = FIELDS.index(p.field)
                cfg.mean[i], cfg.mean_value[i] = 1, p.mean_value
                fields.add(p.field)
            elif isinstance(p, StaticSmagorinskyModel):
                cfg.sgs = 1
                cfg.sgs_dealias, cfg.sgs_p1, cfg.sgs_p2 = _dealias(p.dealiasing)
                cfg.sgs_cs = p.Cs
                cfg.sgs_wall_damping = 1 if p.wall_damping else 0
                cfg.sgs_wall_damping_exponent = float(p.wall_damping_exponent)
                fields.update(FIELDS)
            else:
                raise TypeError(f"unsupported process {p!r}")
        self.fields = [f for f in FIELDS if f in fields]
        cfg.precision = {"fp64": _capi.FP64, "mixed": _capi.MIXED}[precision]
        cfg.device = device
        self._member_arrays = {}
        for name, arr in (("member_cs", member_cs), ("member_z0_lower", member_z0), ("member_source1", member_forcing)):
            if arr is not None:
                a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64))
                if a.shape != (self.members,):
                    raise ValueError(f"{name} needs one value per member")
                self._member_arrays[name] = a
                setattr(cfg, name, a.ctypes.data_as(C.POINTER(C.c_double)))
        self.precision = precision
        self._cfg = cfg
        h = C.c_void_p()
        _capi.check(self._lib.bld_create(C.byref(cfg), C.byref(h)))
        self._h = h
        info = _capi.BldInfo()
        _capi.check(self._lib.bld_get_info(h, C.byref(info)))
        self.info = info
        self._has_sgs = bool(cfg.sgs)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.bld_destroy(h)
            self._h = None

    # -- layout helpers -------------------------------------------------------------
    def nz(self, field):
        return self.n3 - 1 if field == "vel3" else self.n3

    def zeros(self, field):
        return np.zeros((self.nz(field), self.K2, self.K1), dtype=np.complex128)

    def _arrs(self, d):
        out = []
        for f in FIELDS:
            a = d.get(f) if d is not None else None
            if a is None:
                a = self.zeros(f)
            a = np.ascontiguousarray(a, dtype=np.complex128)
            if a.shape != (self.nz(f), self.K2, self.K1):
                raise ValueError(f"{f} has shape {a.shape}, expected {(self.nz(f), self.K2, self.K1)}")
            out.append(a)
        return out

    # -- state ------------------------------------------------------------------------
    def get_state(self, member=0):
        arrs = [self.zeros(f) for f in FIELDS]
        _capi.check(self._lib.bld_get_state(self._h, member, *[a.ctypes.data for a in arrs]))
        return dict(zip(FIELDS, arrs))

    def set_state(self, state, member=0):
        arrs = self._arrs(state)
        _capi.check(self._lib.bld_set_state(self._h, member, *[a.ctypes.data for a in arrs]))

    @property
    def state(self):
        return self.get_state(0)

    # -- the hot path, one call per reference closure ----------------------------------
    def compute_rates(self, state, member=0):
        """``compute_rates!`` + the finite check of ``rate!`` on host arrays."""
        arrs = self._arrs(state)
        rates = [self.zeros(f) for f in FIELDS]
        _capi.check(self._lib.bld_compute_rates(self._h, member, *[a.ctypes.data for a in arrs],
                                                *[r.ctypes.data for r in rates]))
        return dict(zip(FIELDS, rates))

    def apply_projections(self, state, member=0):
        """``apply_projections!`` in place on a dict of host arrays."""
        arrs = self._arrs(state)
        _capi.check(self._lib.bld_apply_projections(self._h, member, *[a.ctypes.data for a in arrs]))
        for f, a in zip(FIELDS, arrs):
            if f in state and state[f] is not None:
                state[f][...] = a
            else:
                state[f] = a
        return state

    # -- physical domain ------------------------------------------------------------------
    @property
    def default_size(self):
        return (2 * self.k1max + 2, 2 * self.k2max + 2)

    def coordinates(self, field="vel1"):
        P1, P2 = self.default_size
        x1 = np.array([self.domain.hsize[0] * float(Fraction(i, P1)) for i in range(P1)])
        x2 = np.array([self.domain.hsize[1] * float(Fraction(i, P2)) for i in range(P2)])
        n = self.n3
        zs = ([Fraction(2 * i - 1, 2 * n) for i in range(1, n + 1)] if field != "vel3"
              else [Fraction(i, n) for i in range(1, n)])
        return x1, x2, np.array([self.domain.vmap(z) for z in zs])

    def set_field(self, field, values, member=0, centered=False):
        """Forward-transform physical values (n3, P2, P1) at the default size into the state
        (``centered``: values at the centres of the grid intervals)."""
        P1, P2 = self.default_size
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(values, dtype=np.float64), (self.nz(field), P2, P1)))
        fn = self._lib.bld_set_field_centered if centered else self._lib.bld_set_field_physical
        _capi.check(fn(self._h, member, FIELDS.index(field), v.ctypes.data))

    def __getitem__(self, field):
        return self.get_field(field)

    def get_field(self, field, member=0, centered=False):
        P1, P2 = self.default_size
        out = np.empty((self.nz(field), P2, P1))
        fn = self._lib.bld_get_field_centered if centered else self._lib.bld_get_field_physical
        _capi.check(fn(self._h, member, FIELDS.index(field), out.ctypes.data))
        return out

    # -- mean profiles on the device --------------------------------------------------------
    def profiles_start(self, on=True):
        _capi.check(self._lib.bld_profiles_start(self._h, 1 if on else 0))

    def profiles_read(self, member=0):
        out = np.zeros(3 * (self.n3 + 1))
        _capi.check(self._lib.bld_profiles_read(self._h, int(member), out.ctypes.data))
        return out

    def profiles_sample(self, member=0):
        out = np.zeros(3 * (self.n3 + 1))
        _capi.check(self._lib.bld_profiles_sample(self._h, int(member), out.ctypes.data))
        return out

    # -- time integration ---------------------------------------------------------------
    def evolve(self, tspan, dt, method=SSPRK33, output=()):
        """``evolve!`` (src/BoundaryLayerDynamics.jl:190-219).  Without output modules
        the whole integration is one call; with them, the steps between output times
        run as graph launches on the device and the modules act at their times."""
        t1, t2 = (0.0, float(tspan)) if np.isscalar(tspan) else (float(tspan[0]), float(tspan[1]))
        if not output:
            _capi.check(self._lib.bld_evolve(self._h, t1, t2, float(dt), _METHODS[method]))
            return self
        if t1 > t2:
            raise ValueError("Integration start time is larger than end time")
        nt = _approxdiv(t2 - t1, dt) if t2 > t1 else 0
        self.prepare()
        for o in output:
            if hasattr(o, "set_dt"):
                o.set_dt(dt)
            o.start(self, t1)
        events = set()
        for o in output:
            for t in o.output_times(t1, t2):
                k = _approxdiv(t - t1, dt)
                if 0 < k <= nt:
                    events.add(k)
        done = 0
        for k in sorted(events | {nt}):
            if k > done:
                self.step(k - done, dt, method)
            t = t2 if k == nt else t1 + k * dt
            for o in output:
                o.at(self, t, k - done)
            done = k
        for o in output:
            o.finish(self, t2)
        return self

    def prepare(self):
        _capi.check(self._lib.bld_prepare(self._h))

    def step(self, nsteps, dt, method=SSPRK33):
        _capi.check(self._lib.bld_step(self._h, int(nsteps), float(dt), _METHODS[method]))

    def sync(self):
        _capi.check(self._lib.bld_sync(self._h))

    def device_state_ptr(self):
        p = C.c_void_p()
        _capi.check(self._lib.bld_state_device_ptr(self._h, C.byref(p)))
        return p.value

    # -- member slots (ensembles and serving) ------------------------------------------
    def set_active(self, mask):
        """Members with a false entry are skipped by every kernel (their state is left as is)."""
        a = np.ascontiguousarray(np.asarray(mask, dtype=np.int32))
        if a.shape != (self.members,):
            raise ValueError("the mask needs one entry per member")
        _capi.check(self._lib.bld_set_active(self._h, a.ctypes.data))

    def set_member_params(self, member, cs=None, z0=None, forcing=None):
        """Replaces a member's Smagorinsky constant, lower roughness length or vel1 forcing."""
        nan = float("nan")
        _capi.check(self._lib.bld_set_member_params(
            self._h, int(member), nan if cs is None else float(cs), nan if z0 is None else float(z0),
            nan if forcing is None else float(forcing)))

    def prepare_member(self, member):
        """Initial projection and right-hand side of one member (the start of ``evolve!``)."""
        _capi.check(self._lib.bld_prepare_member(self._h, int(member)))

    def kernels(self):
        """The kernel variants the autotuner chose (dict)."""
        import json
        buf = C.create_string_buffer(4096)
        _capi.check(self._lib.bld_describe(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def init_random_field(self, field, base, scale, distribution="uniform", seed=0, member=0):
        """Sets ``field`` to base(x3) + scale(x3) r on the device, r uniform on [-1, 1)
        or standard normal from the counter-based generator of ``bld_init_random_field``
        (``workloads.seeded_field`` computes the same values on the host)."""
        nz = self.nz(field)
        b = np.ascontiguousarray(np.broadcast_to(np.asarray(base, float), (nz,)))
        sc = np.ascontiguousarray(np.broadcast_to(np.asarray(scale, float), (nz,)))
        dist = {"uniform": 0, "normal": 1}[distribution]
        _capi.check(self._lib.bld_init_random_field(self._h, int(member), FIELDS.index(field), b.ctypes.data,
                                                    sc.ctypes.data, dist, int(seed) & (2**64 - 1)))

    def progress(self, member=0, tstep=None):
        """The statistics ProgressMonitor reports (src/logging.jl:215-276), computed on
        the device from the member's state, under the reference's labels:
        "Mean Velocity", "Mean KE", "Turbulent KE", "Advective Timescale" (or
        "Adv. Courant Number" with ``tstep``), and with a Smagorinsky wall model
        "Wall Stress τ₁₃" / "Wall Stress τ₂₃" as (lower, upper)."""
        p = _capi.BldProgress()
        _capi.check(self._lib.bld_progress_stats(self._h, int(member), C.byref(p)))
        out = {"Mean Velocity": tuple(p.mean_velocity), "Mean KE": p.mean_ke, "Turbulent KE": p.turbulent_ke}
        if tstep is None:
            out["Advective Timescale"] = p.advective_timescale
        else:
            out["Adv. Courant Number"] = tstep / p.advective_timescale
        if self._has_sgs:
            out["Wall Stress τ₁₃"] = (p.wall_stress[0][0], p.wall_stress[0][1])
            out["Wall Stress τ₂₃"] = (p.wall_stress[1][0], p.wall_stress[1][1])
        return out

    def diverged_members(self):
        """Members whose rates turned non-finite since the last query (clears the record)."""
        out = np.zeros(self.members, dtype=np.int32)
        _capi.check(self._lib.bld_get_diverged(self._h, out.ctypes.data))
        return [int(m) for m in np.flatnonzero(out)]

    def step_async(self, nsteps, dt, method=SSPRK33):
        """Enqueues ``nsteps`` steps on the model's stream without waiting."""
        _capi.check(self._lib.bld_step_async(self._h, int(nsteps), float(dt), _METHODS[method]))

    def idle(self):
        """True when the work enqueued on the model's stream has finished (non-blocking)."""
        v = C.c_int32(0)
        _capi.check(self._lib.bld_stream_idle(self._h, C.byref(v)))
        return bool(v.value)

    @property
    def stream(self):
        p = C.c_void_p()
        _capi.check(self._lib.bld_get_stream(self._h, C.byref(p)))
        return p.value


# --------------------------------------------------------------- API functions (the `!` forms)
def _approxdiv(a, b):
    """approxdiv (src/util.jl): a / b when it is an integer up to rounding, else an error."""
    r = a / b
    ri = round(r)
    if abs(r - ri) > math.sqrt(np.finfo(float).eps) * max(abs(r), abs(ri)):
        raise ValueError("Division has a non-integer result")
    return int(ri)


def initialize(model, path=None, member=0, **initial_conditions):
    """``initialize!(model; vel1=f, ...)`` (src/State.jl:11-31): unspecified fields are zeroed.
    ``initialize(model, path)`` reads a snapshot folder (src/State.jl:33-66)."""
    if path is not None:
        if initial_conditions:
            raise ValueError("initialize from a snapshot path or from initial conditions, not both")
        from .output import initialize_from_snapshot
        initialize_from_snapshot(model, path, member=member)
        return model
    for f in initial_conditions:
        if f not in FIELDS:
            raise KeyError(f"Cannot initialize `{f}`: unknown field")
    P1, P2 = model.default_size
    for f in FIELDS:
        ic = initial_conditions.get(f, 0.0)
        if callable(ic):
            x1, x2, x3 = model.coordinates(f)
            X3, X2, X1 = np.meshgrid(x3, x2, x1, indexing="ij")
            vals = ic(X1, X2, X3)
        else:
            vals = ic
        model.set_field(f, vals, member=member)
    return model


def reset(model):
    """``reset!(model)`` (src/State.jl:68)."""
    for m in range(model.members):
        model.set_state({}, member=m)


def evolve(model, tspan, dt=None, method=SSPRK33, output=()):
    """``evolve!(model, tspan; dt, method, output)`` (src/BoundaryLayerDynamics.jl:190-219)."""
    if dt is None:
        raise ValueError("The keyword argument `dt` is mandatory")
    return model.evolve(tspan, dt, method, output=output)


def coordinates(model, field="vel1"):
    return model.coordinates(field)


def closedchannelflow(Re, dims, **kw):
    """src/BoundaryLayerDynamics.jl:134-138"""
    domain = Domain((4 * math.pi, 2 * math.pi, 2), SmoothWall(), SmoothWall())
    return Model(dims, domain, incompressible_flow(1 / Re, **kw))


def openchannelflow(Re, dims, roughness_length=None, **kw):
    """src/BoundaryLayerDynamics.jl:140-145"""
    wall = SmoothWall() if roughness_length is None else RoughWall(roughness_length)
    domain = Domain((4 * math.pi, 2 * math.pi, 1), wall, FreeSlipBoundary())
    return Model(dims, domain, incompressible_flow(1 / Re, **kw))


from .output import MeanProfiles, ProgressMonitor, Snapshots  # noqa: E402  (output modules for evolve)
