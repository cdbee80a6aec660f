"""CPU oracle for the BoundaryLayerDynamics.jl time-step right-hand side.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` may
import it.  The product (the CUDA library and its host package) never calls
it, and nothing here is a fallback for the GPU path.

It is an FP64 numpy restatement of the reference's algorithm for the path
``rate!`` -> ``compute_rates!`` (linear + physical-domain processes),
``projection!`` -> ``apply_projections!`` (pressure solve, constant mean) and
the explicit integrators (Euler / AB2 / SSPRK22 / SSPRK33).  Every function
cites the reference file:line it follows (paths relative to the
BoundaryLayerDynamics.jl project root).

Third-party arithmetic at the boundary: the reference transforms with FFTW
(``plan_rfft`` / ``plan_brfft``, FFTW.jl 1.4.6 / FFTW_jll 3.3.10 pinned in
``benchmark/Manifest.toml``).  FFTW is not vendored; its published algorithm
(the unnormalised DFT, c2r ignoring the imaginary part of the DC/Nyquist bins)
is restated here through numpy's pocketfft (``norm="forward"`` on the inverse
gives the unnormalised ``brfft``).  Parity is pinned by the reference's own
known-answer tests (``test/*_test.jl``), ported in ``tests/test_oracle_kat.py``;
the reference ships no golden vectors and Julia is not available to run it.

Array layout: a spectral field is complex128 of shape (n3, K2, K1) in C order,
i.e. k1 fastest, then k2 (order 0..k2max, -k2max..-1), then z -- byte-for-byte
the reference's column-major ``Complex{Float64}`` (K1, K2, n3) array
(``src/Grids.jl:74-83,91-93``).  A physical field is float64 (n3, P2, P1),
x fastest, matching the reference's (P1, P2, n3).
"""

from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

__all__ = [
    "Grid", "Domain", "SinusoidalMapping", "SmoothWall", "RoughWall", "FreeSlipBoundary",
    "CustomBoundary", "MomentumAdvection", "MolecularDiffusion", "Pressure", "ConstantSource",
    "ConstantMean", "StaticSmagorinskyModel", "Model", "incompressible_flow", "pdsize",
    "Transform2D", "ODEProblem", "solve", "Euler", "AB2", "SSPRK22", "SSPRK33",
    "set_fft_workers", "DivergenceError", "progress_stats",
]


class DivergenceError(RuntimeError):
    """Raised like ``error("The simulation has diverged.")`` (src/BoundaryLayerDynamics.jl:156)."""


# --------------------------------------------------------------------------------------
# FFT backend (restates FFTW's unnormalised r2c / c2r, src/physical_space.jl:14-21)
# --------------------------------------------------------------------------------------

_FFT = {"workers": 1}


def set_fft_workers(n: int) -> None:
    """Use scipy's pocketfft with ``n`` threads (the CPU baseline uses all host cores)."""
    _FFT["workers"] = max(1, int(n))


def _irfft2_unnormalised(h, s):
    if _FFT["workers"] > 1:
        import scipy.fft as sfft
        return sfft.irfft2(h, s=s, norm="forward", workers=_FFT["workers"])
    return np.fft.irfft2(h, s=s, norm="forward")


def _rfft2_unnormalised(x):
    if _FFT["workers"] > 1:
        import scipy.fft as sfft
        return sfft.rfft2(x, norm="backward", workers=_FFT["workers"])
    return np.fft.rfft2(x, norm="backward")


# --------------------------------------------------------------------------------------
# Grid (src/Grids.jl)
# --------------------------------------------------------------------------------------

class Grid:
    """``StaggeredFourierGrid`` on one process (src/Grids.jl:10-35)."""

    def __init__(self, resolution):
        if isinstance(resolution, int):
            resolution = (resolution, resolution, resolution)
        elif len(resolution) == 2:
            resolution = (resolution[0], resolution[0], resolution[1])
        n1, n2, n3 = (int(r) for r in resolution)
        self.k1max, self.k2max = (n1 - 1) // 2, (n2 - 1) // 2          # :23
        if n3 < 3:                                                      # :28
            raise ValueError("Due to boundary stencils, the grid needs at least 3 vertical layers")
        self.n3global = n3
        self.n3c, self.n3i = n3, n3 - 1                                  # :30-31 (single process)
        self.K1, self.K2 = self.k1max + 1, 2 * self.k2max + 1           # fdsize :91

    def wavenumbers(self, dim):                                         # :74-83
        if dim == 1:
            return np.arange(self.k1max + 1)
        if dim == 2:
            return np.concatenate([np.arange(self.k2max + 1), np.arange(-self.k2max, 0)])
        raise ValueError(f"Invalid dimension `{dim}` for wavenumbers")

    def nz(self, ns):
        return self.n3c if ns == "C" else self.n3i

    def vrange(self, ns, neighbors=False):
        """Rational zeta positions of the C or I nodes (src/Grids.jl:130-141)."""
        n = self.n3global
        zeta = [Fraction(i, 2 * n) for i in range(2 * n + 1)]
        if ns == "C":
            imin = 2 * 1 - (1 if neighbors else 0)
            imax = 2 * n + (1 if neighbors else 0)
        else:
            imin = 2 * 1 + 1 - (1 if neighbors else 0)
            imax = 2 * (1 + self.n3i - 1) + 1 + (1 if neighbors else 0)
        return zeta[imin - 1:imax:2]


NODES = {"vel1": "C", "vel2": "C", "vel3": "I"}                         # src/Grids.jl:97-99


# --------------------------------------------------------------------------------------
# Domain and boundaries (src/Domains.jl)
# --------------------------------------------------------------------------------------

class SmoothWall:
    pass


class RoughWall:
    def __init__(self, roughness, von_karman_constant=0.4):
        self.roughness = roughness
        self.von_karman_constant = von_karman_constant


class FreeSlipBoundary:
    pass


class CustomBoundary:
    """Explicit BCs, e.g. ``CustomBoundary(vel1=("dirichlet", 1.0), vel3="dirichlet")``."""

    def __init__(self, **behaviors):
        self.behaviors = behaviors


def _hasboundarylayer(b):                                               # src/Domains.jl:222-224
    if isinstance(b, (RoughWall, SmoothWall)):
        return True
    if isinstance(b, FreeSlipBoundary):
        return False
    raise ValueError("Could not determine variant of SinusoidalMapping")


class SinusoidalMapping:
    """Grid stretching x3 = sin(zeta*eta*pi/2)/sin(eta*pi/2) (src/Domains.jl:72-130)."""

    def __init__(self, eta, variant="auto"):
        assert 0 < eta < 1
        self.parameter, self.variant = float(eta), variant


def _as_float(z):
    return float(z) if isinstance(z, Fraction) else z


class Domain:
    """``Domain(dims, lower, upper, mapping)`` (src/Domains.jl:30-47,97-135)."""

    def __init__(self, dims, lower_boundary, upper_boundary, mapping=None):
        self.hsize = (float(dims[0]), float(dims[1]))
        if len(dims) == 2:
            x3min, x3max = 0.0, 1.0
        elif isinstance(dims[2], (tuple, list)):
            x3min, x3max = float(dims[2][0]), float(dims[2][1])
        else:
            x3min, x3max = 0.0, float(dims[2])
        self.lower_boundary, self.upper_boundary = lower_boundary, upper_boundary
        self.mapping = mapping
        if mapping is None:                                             # src/Domains.jl:132-133
            l3 = x3max - x3min
            self._vmap = lambda z: x3min + _as_float(z) * l3
            self._dvmap = lambda z: x3max - x3min
        elif isinstance(mapping, SinusoidalMapping):
            assert x3min < x3max
            eta, l = mapping.parameter, x3max - x3min
            variant = mapping.variant
            if variant == "auto":
                bls = (_hasboundarylayer(lower_boundary), _hasboundarylayer(upper_boundary))
                variant = {(True, True): "symmetric", (True, False): "below",
                           (False, True): "above"}.get(bls)
                if variant is None:
                    raise ValueError("Could not determine variant of SinusoidalMapping")
            pi = math.pi
            s = math.sin(eta * pi / 2)
            if variant == "symmetric":
                self._vmap = lambda z: x3min + l / 2 * (1 + math.sin(eta * _as_float(2 * z - 1) * pi / 2) / s)
                self._dvmap = lambda z: l * eta * pi / 2 / s * math.cos(eta * _as_float(2 * z - 1) * pi / 2)
            elif variant == "below":
                self._vmap = lambda z: x3min + l * (1 + math.sin(eta * _as_float(z - 1) * pi / 2) / s)
                self._dvmap = lambda z: l * eta * pi / 2 / s * math.cos(eta * _as_float(z - 1) * pi / 2)
            elif variant == "above":
                self._vmap = lambda z: x3min + l * (math.sin(eta * _as_float(z) * pi / 2) / s)
                self._dvmap = lambda z: l * eta * pi / 2 / s * math.cos(eta * _as_float(z) * pi / 2)
            else:
                raise ValueError("Unknown variant of SinusoidalMapping")
        else:                                                           # custom (x3, dx3) pair
            self._vmap, self._dvmap = mapping

    def vmap(self, zeta):
        return float(self._vmap(zeta))

    def Dvmap(self, zeta):
        return float(self._dvmap(zeta))

    def size3(self):                                                    # src/Domains.jl:50-54
        return self.vmap(Fraction(1)) - self.vmap(Fraction(0))

    def extrema3(self):
        return self.vmap(Fraction(0)), self.vmap(Fraction(1))


def bctype(boundary, field):
    """(kind, value) for ``field`` at ``boundary`` (src/boundary_conditions.jl:85-95,53-59)."""
    if isinstance(boundary, CustomBoundary):
        b = boundary.behaviors[field]
        if isinstance(b, str):
            return (b, 0.0)
        return (b[0], float(b[1]))
    if isinstance(boundary, (SmoothWall, RoughWall)):
        return ("dirichlet", 0.0)
    if isinstance(boundary, FreeSlipBoundary):
        return ("dirichlet", 0.0) if field == "vel3" else ("neumann", 0.0)
    raise ValueError(f"unknown boundary {boundary!r}")


def init_bcs(field, domain, grid):
    """Lower/upper BCs; Neumann keeps gradient*dx3 (src/boundary_conditions.jl:53-79)."""
    out = []
    for b, zeta in ((domain.lower_boundary, 0), (domain.upper_boundary, 1)):
        kind, val = bctype(b, field)
        if kind == "dirichlet":
            out.append(("dirichlet", val))
        elif kind == "neumann":
            dx3 = domain.Dvmap(float(zeta)) / grid.n3global
            out.append(("neumann", val, val * dx3))
        else:
            raise ValueError(f"unsupported boundary behaviour {kind!r}")
    return tuple(out)


def dx1factors(domain, grid):                                           # src/Domains.jl:142-145
    return 1j * grid.wavenumbers(1) * (2 * math.pi / domain.hsize[0])


def dx2factors(domain, grid):
    return 1j * grid.wavenumbers(2) * (2 * math.pi / domain.hsize[1])


def dx3factors(domain, grid, ns, neighbors=False):
    """alpha(zeta) = N3 / (dx3/dzeta) (src/derivatives.jl:10-19)."""
    a = lambda z: grid.n3global / domain.Dvmap(float(z))
    zeta = grid.vrange(ns)
    if neighbors:
        znb = grid.vrange(ns, neighbors=True)
        return [(a(znb[i]), a(zeta[i]), a(znb[i + 1])) for i in range(len(zeta))]
    return np.array([a(z) for z in zeta])


# --------------------------------------------------------------------------------------
# Physical-domain sizes and transforms (src/physical_space.jl)
# --------------------------------------------------------------------------------------

def _pdsize_quadratic(kmax):                                            # :49-56
    if math.log2(1 + kmax).is_integer():
        return 3 * kmax + 3
    return 3 * kmax + (1 if kmax % 2 == 1 else 2)


def pdsize(grid, dealiasing=None):                                      # :42-56
    if dealiasing is None:
        return (2 + 2 * grid.k1max, 2 + 2 * grid.k2max)
    if isinstance(dealiasing, tuple):
        return tuple(int(d) for d in dealiasing)
    if dealiasing == "quadratic":
        return (_pdsize_quadratic(grid.k1max), _pdsize_quadratic(grid.k2max))
    raise ValueError(f"Unsupported dealiasing type: {dealiasing}")


class Transform2D:
    """Padded/truncated 2-D transforms of whole fields, layer by layer.

    ``get_field`` follows get_layer!/get_field! (src/physical_space.jl:277-312);
    ``add_field`` follows add_layer!/add_field! (src/physical_space.jl:208-246).
    """

    def __init__(self, grid, dims):
        self.P1, self.P2 = int(dims[0]), int(dims[1])
        self.K1, self.K2 = grid.K1, grid.K2
        self.k1m = min(self.P1 // 2 + 1, self.K1) - 1                   # :280
        self.k2m = (min(self.P2, self.K2) - 1) // 2                     # :281

    def get_field(self, fd, prefactors=None, centered=False):
        nz = fd.shape[0]
        k1m, k2m, P1, P2 = self.k1m, self.k2m, self.P1, self.P2
        src = fd if prefactors is None else fd * prefactors
        h = np.zeros((nz, P2, P1 // 2 + 1), dtype=np.complex128)
        h[:, :k2m + 1, :k1m + 1] = src[:, :k2m + 1, :k1m + 1]           # :283-285
        if k2m > 0:
            h[:, P2 - k2m:, :k1m + 1] = src[:, self.K2 - k2m:, :k1m + 1]  # :286-288
        if centered:
            h = h * half_shift_factors(P1, P2, +1)                      # :291
        return _irfft2_unnormalised(h, (P2, P1))                        # :293

    def add_field(self, fd, pd, prefactors=None, centered=False):
        k1m, k2m, P1, P2 = self.k1m, self.k2m, self.P1, self.P2
        x = _rfft2_unnormalised(pd)                                     # :222
        if centered:
            x = x * half_shift_factors(P1, P2, -1)                      # :223
        f = 1 / (P1 * P2)                                               # :219
        if prefactors is not None:                                      # (1,K1) or (K2,1) broadcast
            pr = np.asarray(prefactors)
            cols = slice(None) if pr.shape[1] == 1 else slice(0, k1m + 1)
            lo = slice(None) if pr.shape[0] == 1 else slice(0, k2m + 1)
            hi = slice(None) if pr.shape[0] == 1 else slice(self.K2 - k2m, None)
        a = x[:, :k2m + 1, :k1m + 1] * f
        if prefactors is not None:
            a = a * pr[lo, cols]
        fd[:, :k2m + 1, :k1m + 1] += a                                  # :225-227
        if k2m > 0:
            b = x[:, P2 - k2m:, :k1m + 1] * f
            if prefactors is not None:
                b = b * pr[hi, cols]
            fd[:, self.K2 - k2m:, :k1m + 1] += b                        # :228-230
        return fd

    def set_field(self, fd, pd, centered=False):                        # :253-256
        fd[...] = 0
        return self.add_field(fd, pd, centered=centered)


def half_shift_factors(P1, P2, sign):
    """shift!/unshift! (src/physical_space.jl:321-336): exp(sign i pi (k1/P1 + k2/P2))
    on the (P2, P1/2+1) half spectrum, the Nyquist row counted as negative."""
    k1 = np.arange(P1 // 2 + 1)
    i2 = np.arange(1, P2 + 1)
    k2 = np.where(2 * i2 > P2, i2 - P2 - 1, i2 - 1)
    return np.exp(sign * 1j * np.pi * (k1[None, :] / P1 + k2[:, None] / P2))[None, :, :]


# --------------------------------------------------------------------------------------
# Output: CBD files (src/fileio.jl) and mean profiles (src/logging.jl:333-491)
# --------------------------------------------------------------------------------------

CBD_MAGIC = bytes.fromhex("CBDF")


def writecbd(dtype, filename, field, x1, x2, x3, xmin, xmax):
    """writecbd (src/fileio.jl:26-62): identifier, sizes, limits, coordinates, data
    (x1 fastest).  ``field`` is indexed [x3][x2][x1]."""
    import struct
    dtype = np.dtype(dtype)
    n3, n2, n1 = np.shape(field)
    ident = bytes([0xCB, 0xDF, 1, 0, 0, 0, 0, dtype.itemsize])        # :29-32
    with open(filename, "wb") as f:
        f.write(ident)
        f.write(struct.pack("<3Q", n1, n2, n3))                          # :44
        f.write(struct.pack("<3d", *xmin))                               # :45
        f.write(struct.pack("<3d", *xmax))                               # :46
        f.write(struct.pack(f"<{n1}d", *x1))                             # :47
        f.write(struct.pack(f"<{n2}d", *x2))                             # :48
        f.write(struct.pack(f"<{n3}d", *x3))                             # :54
        f.write(np.asarray(field, dtype=dtype.newbyteorder("<")).tobytes())  # :59


def readcbd(filename):
    """readcbd (src/fileio.jl:64-108) for the whole x3 range."""
    import struct
    with open(filename, "rb") as f:
        ident = f.read(8)
        assert ident[:2] == CBD_MAGIC and ident[2] == 1
        dtype = {4: np.dtype("<f4"), 8: np.dtype("<f8")}[ident[7]]
        n1, n2, n3 = struct.unpack("<3Q", f.read(24))
        xmin = struct.unpack("<3d", f.read(24))
        xmax = struct.unpack("<3d", f.read(24))
        x1 = np.array(struct.unpack(f"<{n1}d", f.read(8 * n1)))
        x2 = np.array(struct.unpack(f"<{n2}d", f.read(8 * n2)))
        x3 = np.array(struct.unpack(f"<{n3}d", f.read(8 * n3)))
        data = np.frombuffer(f.read(), dtype=dtype).reshape(n3, n2, n1)
    return xmin, xmax, x1, x2, x3, data


class MeanProfiles:
    """Time-averaged horizontal means (MeanProfiles, src/logging.jl:333-491): one
    sample per checkpoint (every step), trapezoidal rule in time, vel3 profiles
    with their two boundary entries (zero for state samples)."""

    def __init__(self, n3, t1, profiles=("vel1", "vel2", "vel3")):
        size = lambda f: n3 + 1 if f == "vel3" else n3                  # :351-353
        self.means = {f: np.zeros(size(f)) for f in profiles}
        self.samples = {f: np.zeros(size(f)) for f in profiles}
        self.timespan = [t1, t1]
        self.intervals = 0

    def sample_state(self, state):                                      # :380-413
        for f in self.samples:
            col = state[f][:, 0, 0].real                                # hmean, :411
            if f == "vel3":
                self.samples[f][1:-1] = col
            else:
                self.samples[f][:] = col

    def step(self, state, t):
        """prepare_samples! + log_state! + process_log! for a checkpoint at t."""
        w = (t - self.timespan[1]) / 2                                  # :373
        for f in self.means:
            self.means[f] += w * self.samples[f]
        self.sample_state(state)
        for f in self.means:                                            # :434-437
            self.means[f] += w * self.samples[f]
        self.timespan[1] = t
        self.intervals += 1

    def averages(self):                                                 # :461-467
        dt = self.timespan[1] - self.timespan[0]
        return {f: v / dt for f, v in self.means.items()}


def progress_stats(model, state=None, tstep=None):
    """The statistics ProgressMonitor prints (src/logging.jl:215-266), from the
    state of ``model``: "Mean Velocity" (log_state! for the NamedTuple state,
    :240-247), "Mean KE" / "Turbulent KE" and the advective time scale (or Courant
    number) from the physical fields of the largest physical-domain size
    (log_state! for the Dict of physical fields, :249-276, ``largest`` :206-211),
    and the mean wall-model stresses of the SGS model (log_sample!, :230-237;
    stress_bc, src/processes/static_smagorinsky.jl:195-200; hmean,
    src/logging.jl:411-413)."""
    state = model.state if state is None else state
    g, dom = model.grid, model.domain
    n = g.n3global
    L3 = dom.size3()
    dzeta = Fraction(1, n)
    dx3c = np.array([float(dzeta) * dom.Dvmap(z) for z in g.vrange("C")])       # :164-165
    dx3i = np.array([float(dzeta) * dom.Dvmap(z) for z in g.vrange("I")])
    out = {"Mean Velocity": tuple(float(np.sum(np.real(state[f][:, 0, 0]) * w / L3))
                                  for f, w in (("vel1", dx3c), ("vel2", dx3c), ("vel3", dx3i)))}
    dims = []
    for p in model.processes:
        if isinstance(p, (_DiscretizedAdvection, _DiscretizedSmagorinsky)):
            dims.append(tuple(p.dims))
    big = max(dims) if dims else pdsize(g)
    tf = model.transform(big)
    u, v, w = (tf.get_field(state[f]) for f in ("vel1", "vel2", "vel3"))
    ub, vb = u.mean(axis=(1, 2)), v.mean(axis=(1, 2))
    mke = ub ** 2 + vb ** 2
    ke = (u ** 2).mean(axis=(1, 2)) + (v ** 2).mean(axis=(1, 2))
    out["Mean KE"] = float(np.sum(mke))
    out["Turbulent KE"] = float(np.sum(ke - mke))
    wmax = np.abs(w).max(axis=(1, 2))
    with np.errstate(divide="ignore"):
        dtmin = float(np.min(dx3i / wmax)) if len(wmax) else math.inf
    if tstep is None:
        out["Advective Timescale"] = dtmin
    else:
        out["Adv. Courant Number"] = tstep / dtmin
    for p in model.processes:
        if isinstance(p, _DiscretizedSmagorinsky):
            ts = model.transform(tuple(p.dims))
            us, vs = ts.get_field(state["vel1"]), ts.get_field(state["vel2"])
            taus = []
            for i in (0, 1):
                vals = []
                for side, layer in ((0, 0), (1, -1)):
                    if p.wall_dynamic[side]:
                        uu, vv = us[layer], vs[layer]
                        vel = uu if i == 0 else vv
                        vals.append(float(np.mean(p.factors_stress[side] * vel * np.sqrt(uu ** 2 + vv ** 2))))
                    else:
                        vals.append(0.0)                                # ConstantValue(0) at a free-slip wall
                taus.append(tuple(vals))
            out["Wall Stress τ₁₃"], out["Wall Stress τ₂₃"] = taus
    return out


def h1range(P, centered=False):                                         # src/physical_space.jl:64-65
    return [Fraction(2 * i + (1 if centered else 0), 2 * P) for i in range(P)]


# --------------------------------------------------------------------------------------
# Vertical stencils on layer stacks (src/derivatives.jl:103-138)
# --------------------------------------------------------------------------------------

def dx3_c2i(term, D3i):
    """I-layer i = -D3i[i]*C[i] + D3i[i]*C[i+1] (src/derivatives.jl:104-110,121)."""
    d = D3i.reshape(-1, 1, 1)
    return -d * term[:-1] + d * term[1:]


def dx3_i2c_physical(term, lower, upper, D3c):
    """C-layer i from I-layers (lbc, I..., ubc), physical domain (src/derivatives.jl:111-138).

    ``lower``/``upper`` are either a scalar Dirichlet value or a per-point array
    (``DynamicValues``); both enter as ``-D3*below + D3*above``.
    """
    d = D3c.reshape(-1, 1, 1)
    n = term.shape[0] + 1
    out = np.empty((n,) + term.shape[1:])
    out[0] = -d[0] * lower + d[0] * term[0]
    out[1:n - 1] = -d[1:n - 1] * term[:-1] + d[1:n - 1] * term[1:]
    out[n - 1] = -d[n - 1] * term[-1] + d[n - 1] * upper
    return out


# --------------------------------------------------------------------------------------
# Process definitions (constructors mirror the reference keywords)
# --------------------------------------------------------------------------------------

class MomentumAdvection:                                                # src/processes/momentum_advection.jl:18-21
    def __init__(self, dealiasing="quadratic"):
        self.dealiasing = dealiasing


class MolecularDiffusion:                                               # src/processes/molecular_diffusion.jl:13-19
    def __init__(self, field, diffusivity):
        self.field, self.diffusivity = field, float(diffusivity)


class Pressure:                                                         # src/processes/pressure.jl:215-218
    def __init__(self, batch_size=64):
        self.batch_size = batch_size


class ConstantSource:                                                   # src/processes/sources.jl:13-17
    def __init__(self, field, strength=1):
        self.field, self.strength = field, float(strength)


class ConstantMean:                                                     # src/processes/sources.jl:47-51
    def __init__(self, field, mean_value=1):
        self.field, self.mean_value = field, float(mean_value)


class StaticSmagorinskyModel:                                           # src/processes/static_smagorinsky.jl:15-22
    def __init__(self, dealiasing=None, Cs=0.1, wall_damping=True, wall_damping_exponent=2):
        self.dealiasing, self.model_constant = dealiasing, float(Cs)
        self.wall_damping, self.wall_damping_exponent = wall_damping, wall_damping_exponent


def incompressible_flow(viscosity, sgs_model=None, constant_forcing=None, constant_flux=None):
    """Process list of ``incompressible_flow`` (src/BoundaryLayerDynamics.jl:116-132)."""
    if constant_flux is not None and constant_forcing is not None:
        raise ValueError("Momentum source set up for both constant forcing and constant flux")
    if constant_flux is None and constant_forcing is None:
        constant_forcing = 1
    procs = [MomentumAdvection()]
    procs += [MolecularDiffusion(v, viscosity) for v in ("vel1", "vel2", "vel3")]
    procs.append(Pressure())
    vel = ("vel1", "vel2")
    if constant_forcing is not None:
        vals = constant_forcing if isinstance(constant_forcing, (tuple, list)) else (constant_forcing,)
        procs += [ConstantSource(vel[i], f) for i, f in enumerate(vals)]
    else:
        vals = constant_flux if isinstance(constant_flux, (tuple, list)) else (constant_flux,)
        procs += [ConstantMean(vel[i], m) for i, m in enumerate(vals)]
    if sgs_model is not None:
        procs.append(sgs_model)
    return procs


# --------------------------------------------------------------------------------------
# Discretised processes
# --------------------------------------------------------------------------------------

class _DiscretizedDiffusion:
    """src/processes/molecular_diffusion.jl:31-72 with layers_expand_full
    (src/boundary_conditions.jl:254-359) and second_derivatives (src/derivatives.jl:21-27)."""

    kind = "linear"

    def __init__(self, d, domain, grid):
        self.field, self.nu = d.field, d.diffusivity
        self.ns = NODES[d.field]
        self.bcs = init_bcs(d.field, domain, grid)
        k1, k2 = grid.wavenumbers(1), grid.wavenumbers(2)
        self.DD1 = (-k1 ** 2 * (2 * math.pi / domain.hsize[0]) ** 2).reshape(1, -1)
        self.DD2 = (-k2 ** 2 * (2 * math.pi / domain.hsize[1]) ** 2).reshape(-1, 1)
        self.DD3 = dx3factors(domain, grid, self.ns, neighbors=True)

    def _expanded(self, q):
        """Layers (below, q..., above) (src/boundary_conditions.jl:263-359)."""
        lower, upper = self.bcs
        n = q.shape[0]
        if self.ns == "I":
            for bc in (lower, upper):
                if bc[0] != "dirichlet":
                    raise ValueError("I-node diffusion supports Dirichlet boundaries only")
            return lower[1], list(q), upper[1]          # scalar values, broadcast to every mode
        if lower[0] == "dirichlet":
            below = (-15 * q[0] + 5 * q[1] - q[2]) / 5                  # src/boundary_conditions.jl:294-295
            below[0, 0] += 16 * lower[1] / 5
        else:
            below = (21 * q[0] + 3 * q[1] - q[2]) / 23                  # src/boundary_conditions.jl:330-331
            below[0, 0] -= 24 * lower[2] / 23
        if upper[0] == "dirichlet":
            above = (-15 * q[n - 1] + 5 * q[n - 2] - q[n - 3]) / 5      # src/boundary_conditions.jl:312-313
            above[0, 0] += 16 * upper[1] / 5
        else:
            above = (21 * q[n - 1] + 3 * q[n - 2] - q[n - 3]) / 23      # src/boundary_conditions.jl:348-349
            above[0, 0] -= 24 * (-upper[2]) / 23
        return below, list(q), above

    def add_rates(self, rates, state):
        q = state[self.field]
        below, layers, above = self._expanded(q)
        ext = [below] + layers + [above]
        out = rates[self.field]
        for i in range(q.shape[0]):                                     # src/processes/molecular_diffusion.jl:59-61
            a, b, c = self.DD3[i]
            out[i] += self.nu * (a * b * ext[i] + (self.DD1 + self.DD2 - a * b - b * c) * ext[i + 1]
                                 + b * c * ext[i + 2])


class _DiscretizedSource:
    """ConstantSource.add_rates! (src/processes/sources.jl:32-35)."""

    kind = "linear"

    def __init__(self, d, domain, grid):
        self.field, self.strength = d.field, d.strength

    def add_rates(self, rates, state):
        rates[self.field][:, 0, 0] += self.strength


class _DiscretizedConstantMean:
    """ConstantMean projection (src/processes/sources.jl:60-77)."""

    kind = "projection"

    def __init__(self, d, domain, grid):
        if NODES[d.field] != "C":
            raise ValueError("The constant-mean source currently does not handle I-nodes correctly")
        self.field, self.mean_value = d.field, d.mean_value
        self.weight = 1 / dx3factors(domain, grid, "C") / domain.size3()

    def apply_projection(self, state):
        f = state[self.field]
        current = 0.0
        for i in range(f.shape[0]):
            current += f[i, 0, 0].real * self.weight[i]
        f[:, 0, 0] += self.mean_value - current


def ldlt_factor(diag, offdiag):
    """gamma of the batched LDL^T factorisation (src/processes/pressure.jl:85-95).

    ``diag`` has shape (..., n); ``offdiag`` (n-1,) or (..., n-1).
    """
    diag = np.asarray(diag, dtype=np.float64)
    beta = np.broadcast_to(np.asarray(offdiag, dtype=np.float64), diag.shape[:-1] + (diag.shape[-1] - 1,))
    gamma = np.empty_like(diag)
    gamma[..., 0] = 1 / diag[..., 0]
    for z in range(1, diag.shape[-1]):
        gamma[..., z] = 1 / (diag[..., z] - gamma[..., z - 1] * beta[..., z - 1] ** 2)
    return gamma


def ldlt_solve(gamma, offdiag, rhs):
    """In-place ldiv! with symthomas_batch_fwd!/bwd! (src/processes/pressure.jl:106-201).

    ``rhs`` has shape (n, ...) (z slowest, like a field); ``gamma`` (..., n).
    """
    n = rhs.shape[0]
    beta = np.broadcast_to(np.asarray(offdiag, dtype=np.float64), gamma.shape[:-1] + (n - 1,))
    rhs[0] = gamma[..., 0] * rhs[0]
    for z in range(1, n):
        rhs[z] = gamma[..., z] * (rhs[z] - beta[..., z - 1] * rhs[z - 1])
    for z in range(n - 2, -1, -1):
        rhs[z] = rhs[z] - gamma[..., z] * beta[..., z] * rhs[z + 1]
    return rhs


class _DiscretizedPressure:
    """Pressure projection (src/processes/pressure.jl:38-426)."""

    kind = "projection"

    def __init__(self, d, domain, grid):
        n = grid.n3global
        self.offdiag = dx3factors(domain, grid, "I")                    # :234
        aC = dx3factors(domain, grid, "C")                              # :238
        self.aC, self.aI = aC, self.offdiag
        # d3g3 diagonal (:267-275)
        ai_ext = np.array([n / domain.Dvmap(float(z)) for z in grid.vrange("C", neighbors=True)])
        d3g3 = np.zeros(n)
        d3g3[1:] -= ai_ext[1:n]
        d3g3[:n - 1] -= ai_ext[1:n]
        k1, k2 = grid.wavenumbers(1), grid.wavenumbers(2)
        s1, s2 = 1 / domain.hsize[0], 1 / domain.hsize[1]               # scalefactor (src/Domains.jl:160-171)
        K2, K1 = grid.K2, grid.K1
        diag = np.empty((K2, K1, n))
        for j in range(K2):
            for i in range(K1):
                if k1[i] == 0 and k2[j] == 0:                           # :240, adjust_d3g3_diagonal :287-296
                    dv = d3g3.copy()
                    last_ev = n / domain.Dvmap(float(grid.vrange("C", neighbors=True)[-2]))
                    dv[-1] = -3 * last_ev
                else:
                    dv = np.array([d3g3[z] - 4 * math.pi ** 2 * (k1[i] ** 2 * s1 ** 2 + k2[j] ** 2 * s2 ** 2) / aC[z]
                                   for z in range(n)])
                diag[j, i] = dv
        self.diag = diag
        self.gamma = ldlt_factor(diag, self.offdiag)
        self.D1 = dx1factors(domain, grid).reshape(1, -1)
        self.D2 = dx2factors(domain, grid).reshape(-1, 1)
        self.bc3 = init_bcs("vel3", domain, grid)

    def solve(self, rhs):
        return ldlt_solve(self.gamma, self.offdiag, rhs)

    def pressure(self, state):
        """solve_pressure! (src/processes/pressure.jl:334-361)."""
        lbc, ubc = self.bc3
        if lbc[0] != "dirichlet" or ubc[0] != "dirichlet":
            raise ValueError("The pressure solver only supports Dirichlet BCs")
        u1, u2, u3 = state["vel1"], state["vel2"], state["vel3"]
        n = u1.shape[0]
        p = np.empty_like(u1)
        for i in range(n):                                              # div! :368-378
            h = 1 / self.aC[i]
            val = u1[i] * self.D1 * h + u2[i] * self.D2 * h
            if i == 0:
                val = val + u3[0]
                val[0, 0] -= lbc[1]
            elif i == n - 1:
                val = val - u3[n - 2]
                val[0, 0] += ubc[1]
            else:
                val = val - u3[i - 1] + u3[i]
            p[i] = val
        if lbc[1] != ubc[1]:
            raise ValueError("The mean flow must be equal at both vertical boundaries.")
        p[n - 1, 0, 0] = 0                                              # adjust_pressure_rhs! :396
        return self.solve(p)

    def apply_projection(self, state):                                  # :300-305, add_gradient! :405-426
        p = self.pressure(state)
        state["vel1"] += -1 * self.D1 * p
        state["vel2"] += -1 * self.D2 * p
        d = self.aI.reshape(-1, 1, 1)
        state["vel3"] += -1 * (-d * p[:-1] + d * p[1:])
        return p


class _DiscretizedAdvection:
    """MomentumAdvection in rotation form (src/processes/momentum_advection.jl:31-206)."""

    kind = "nonlinear"

    def __init__(self, d, domain, grid):
        self.dims = pdsize(grid, d.dealiasing)
        self.bc3 = init_bcs("vel3", domain, grid)
        self.D1 = dx1factors(domain, grid).reshape(1, -1)
        self.D2 = dx2factors(domain, grid).reshape(-1, 1)
        self.D3i = dx3factors(domain, grid, "I").reshape(-1, 1, 1)

    def vorticity(self, state):
        """Frequency-domain vorticity (src/derivatives.jl:198-230)."""
        u, v, w = state["vel1"], state["vel2"], state["vel3"]
        D1, D2, D3 = self.D1, self.D2, self.D3i
        vort1 = D2 * w - (-D3 * v[:-1] + D3 * v[1:])
        vort2 = (-D3 * u[:-1] + D3 * u[1:]) - D1 * w
        vort3 = D1 * v - D2 * u
        return vort1, vort2, vort3

    def add_psrates(self, psrates, state, tf):
        for bc in self.bc3:
            if bc[0] != "dirichlet":
                raise ValueError("Advection requires Dirichlet boundary conditions for vel3")
            if bc[1] != 0:
                raise ValueError("Advection for non-zero w at boundary not implemented")
        u = tf.get_field(state["vel1"])
        v = tf.get_field(state["vel2"])
        w = tf.get_field(state["vel3"])
        o1, o2, o3 = (tf.get_field(x) for x in self.vorticity(state))
        n = u.shape[0]
        adv1 = np.empty_like(u)
        adv2 = np.empty_like(u)
        # :179-203 (interior, lower and upper layer forms)
        adv1[0] = o3[0] * v[0] - 0.5 * (o2[0] * w[0])
        adv2[0] = 0.5 * (o1[0] * w[0]) - o3[0] * u[0]
        adv1[1:n - 1] = o3[1:n - 1] * v[1:n - 1] - 0.5 * (o2[:n - 2] * w[:n - 2] + o2[1:n - 1] * w[1:n - 1])
        adv2[1:n - 1] = 0.5 * (o1[:n - 2] * w[:n - 2] + o1[1:n - 1] * w[1:n - 1]) - o3[1:n - 1] * u[1:n - 1]
        adv1[n - 1] = o3[n - 1] * v[n - 1] - 0.5 * (o2[n - 2] * w[n - 2])
        adv2[n - 1] = 0.5 * (o1[n - 2] * w[n - 2]) - o3[n - 1] * u[n - 1]
        adv3 = o2 * 0.5 * (u[:-1] + u[1:]) - o1 * 0.5 * (v[:-1] + v[1:])  # :206
        psrates["vel1"] += adv1
        psrates["vel2"] += adv2
        psrates["vel3"] += adv3

    def rate_names(self):
        return ("vel1", "vel2", "vel3")


class _DiscretizedSmagorinsky:
    """Static Smagorinsky SGS model with wall model (src/processes/static_smagorinsky.jl:44-249)."""

    kind = "nonlinear"

    def __init__(self, d, domain, grid):
        self.dims = pdsize(grid, d.dealiasing)
        n = grid.n3global
        d1 = domain.hsize[0] / (2 * grid.k1max + 2)                     # src/processes/static_smagorinsky.jl:54-55
        d2 = domain.hsize[1] / (2 * grid.k2max + 2)
        zc, zi = grid.vrange("C"), grid.vrange("I")
        d3c = np.array([domain.Dvmap(z) for z in zc]) / n               # src/processes/static_smagorinsky.jl:56-57
        d3i = np.array([domain.Dvmap(z) for z in zi]) / n
        lc = d.model_constant * np.cbrt(d1 * d2 * d3c)                  # src/processes/static_smagorinsky.jl:58-59
        li = d.model_constant * np.cbrt(d1 * d2 * d3i)
        if d.wall_damping:                                              # src/processes/static_smagorinsky.jl:61-85
            x3c = np.array([domain.vmap(z) for z in zc])
            x3i = np.array([domain.vmap(z) for z in zi])
            x3min, x3max = domain.extrema3()
            lcw = np.array([self._mixing_length(x, x3min, x3max, domain) for x in x3c])
            liw = np.array([self._mixing_length(x, x3min, x3max, domain) for x in x3i])
            N = d.wall_damping_exponent
            lc = (lc ** (-N) + lcw ** (-N)) ** (-1 / N)
            li = (li ** (-N) + liw ** (-N)) ** (-1 / N)
        self.lc, self.li = lc.reshape(-1, 1, 1), li.reshape(-1, 1, 1)
        x3min, x3max = domain.extrema3()
        dx3_below = domain.vmap(zc[0]) - x3min                          # src/processes/static_smagorinsky.jl:99-100
        dx3_above = x3max - domain.vmap(zc[-1])
        lw = self._init_wall(domain.lower_boundary, dx3_below)
        uw = self._init_wall(domain.upper_boundary, dx3_above)
        self.wall_dynamic = (lw[0], uw[0])
        self.factors_strain = (lw[1], -uw[1])                           # src/processes/static_smagorinsky.jl:106-107
        self.factors_stress = (lw[2], -uw[2])
        self.D3c = dx3factors(domain, grid, "C")
        self.D3i = dx3factors(domain, grid, "I")
        self.D1 = dx1factors(domain, grid).reshape(1, -1)
        self.D2 = dx2factors(domain, grid).reshape(-1, 1)
        self.bc3 = init_bcs("vel3", domain, grid)

    @staticmethod
    def _mixing_length(x3, x3min, x3max, domain):                       # :125-127
        def ml(dist, wall):
            if isinstance(wall, FreeSlipBoundary):
                return math.inf
            if isinstance(wall, RoughWall):
                return dist * wall.von_karman_constant
            raise ValueError("SGS model only supports rough-wall and free-slip boundaries")
        return min(ml(x3 - x3min, domain.lower_boundary), ml(x3max - x3, domain.upper_boundary))

    @staticmethod
    def _init_wall(boundary, dx3):                                      # src/processes/static_smagorinsky.jl:92-98
        if isinstance(boundary, RoughWall):
            lg = math.log(dx3 / boundary.roughness)
            return (True, 1 / (2 * dx3 * lg), -boundary.von_karman_constant ** 2 / lg ** 2)
        if isinstance(boundary, FreeSlipBoundary):
            return (False, 0.0, 0.0)
        raise ValueError("SGS model only supports rough-wall and free-slip boundaries")

    def terms(self, state, tf):
        """Physical-domain terms (src/processes/static_smagorinsky.jl:39-42, src/derivatives.jl:32-101,235-241)."""
        vel1 = tf.get_field(state["vel1"])
        vel2 = tf.get_field(state["vel2"])
        vel3 = tf.get_field(state["vel3"])
        vel1_1 = tf.get_field(state["vel1"], self.D1)
        vel1_2 = tf.get_field(state["vel1"], self.D2)
        vel2_1 = tf.get_field(state["vel2"], self.D1)
        vel2_2 = tf.get_field(state["vel2"], self.D2)
        vel3_1 = tf.get_field(state["vel3"], self.D1)
        vel3_2 = tf.get_field(state["vel3"], self.D2)
        lbc, ubc = self.bc3
        if lbc[0] != "dirichlet" or ubc[0] != "dirichlet":
            raise ValueError("only Dirichlet vel3 boundaries are supported for vel3_3")
        vel3_3 = dx3_i2c_physical(vel3, lbc[1], ubc[1], self.D3c)
        vel1_3 = dx3_c2i(vel1, self.D3i)
        vel2_3 = dx3_c2i(vel2, self.D3i)
        s12 = (vel1_2 + vel2_1) / 2
        s13 = (vel1_3 + vel3_1) / 2
        s23 = (vel2_3 + vel3_2) / 2
        return dict(vel1=vel1, vel2=vel2, s11=vel1_1, s22=vel2_2, s33=vel3_3, s12=s12, s13=s13, s23=s23)

    def _wall_values(self, vel_c, factors, side):
        """strain_bc/stress_bc: DynamicValues at the wall-adjacent C layer, or ConstantValue(0)."""
        return None if not self.wall_dynamic[side] else factors[side] * vel_c

    def total_strain(self, t):
        """total_strain! (src/processes/static_smagorinsky.jl:202-233)."""
        s11, s22, s33, s12, s13, s23 = t["s11"], t["s22"], t["s33"], t["s12"], t["s13"], t["s23"]
        sc = s11 ** 2 + s22 ** 2 + s33 ** 2 + 2 * s12 ** 2
        si = 2 * s13 ** 2 + 2 * s23 ** 2
        for s, cnt in ((s11, 1), (s22, 1), (s33, 1), (s12, 2)):        # add_interpolated_sq! :240
            si += cnt * (s[:-1] + s[1:]) ** 2 / 4
        n = sc.shape[0]
        for s, vel in ((s13, t["vel1"]), (s23, t["vel2"])):
            lo = self._wall_values(vel[0], self.factors_strain, 0)
            hi = self._wall_values(vel[n - 1], self.factors_strain, 1)
            # layers (lbc, I..., ubc); dynamic values are not interpolated (:245-249)
            sc[0] += 2 * lo ** 2 if lo is not None else 2 * (0.0 + s[0]) ** 2 / 4
            sc[1:n - 1] += 2 * (s[:-1] + s[1:]) ** 2 / 4
            sc[n - 1] += 2 * hi ** 2 if hi is not None else 2 * (s[n - 2] + 0.0) ** 2 / 4
        return np.sqrt(2 * sc), np.sqrt(2 * si)

    def add_psrates(self, psrates, state, tf):
        """add_rates! (src/processes/static_smagorinsky.jl:129-192)."""
        t = self.terms(state, tf)
        evc, evi = self.total_strain(t)
        evc = evc * self.lc ** 2
        evi = evi * self.li ** 2
        self.eddyviscosity_c, self.eddyviscosity_i = evc, evi
        n = evc.shape[0]
        sgsc = -2 * evc * t["s11"]
        psrates["vel1_1"] -= sgsc
        sgsc = -2 * evc * t["s22"]
        psrates["vel2_2"] -= sgsc
        sgsc = -2 * evc * t["s33"]
        psrates["vel3"] -= dx3_c2i(sgsc, self.D3i)
        sgsc = -2 * evc * t["s12"]
        psrates["vel1_2"] -= sgsc
        psrates["vel2_1"] -= sgsc
        u_lo, u_hi = t["vel1"][0], t["vel1"][n - 1]
        v_lo, v_hi = t["vel2"][0], t["vel2"][n - 1]
        for comp, key, rate_h, rate_c in ((1, "s13", "vel3_1", "vel1"), (2, "s23", "vel3_2", "vel2")):
            sgsi = -2 * evi * t[key]
            psrates[rate_h] -= sgsi
            bcs = []
            for side, (a, b) in enumerate(((u_lo, v_lo), (u_hi, v_hi))):   # stress_bc :195-200
                if self.wall_dynamic[side]:
                    vel = a if comp == 1 else b
                    bcs.append(self.factors_stress[side] * vel * np.sqrt(a ** 2 + b ** 2))
                else:
                    bcs.append(0.0)
            psrates[rate_c] -= dx3_i2c_physical(sgsi, bcs[0], bcs[1], self.D3c)

    def rate_names(self):
        return ("vel1", "vel1_1", "vel1_2", "vel2", "vel2_1", "vel2_2", "vel3", "vel3_1", "vel3_2")


# --------------------------------------------------------------------------------------
# Model (src/BoundaryLayerDynamics.jl, src/Processes.jl)
# --------------------------------------------------------------------------------------

_DISCRETIZE = {
    MomentumAdvection: _DiscretizedAdvection,
    MolecularDiffusion: _DiscretizedDiffusion,
    Pressure: _DiscretizedPressure,
    ConstantSource: _DiscretizedSource,
    ConstantMean: _DiscretizedConstantMean,
    StaticSmagorinskyModel: _DiscretizedSmagorinsky,
}


def _flatten(procs):
    for p in procs:
        if isinstance(p, (list, tuple)):
            yield from _flatten(p)
        else:
            yield p


class Model:
    """``Model(resolution, domain, processes)`` (src/BoundaryLayerDynamics.jl:72-97)."""

    def __init__(self, resolution, domain, processes):
        self.domain, self.grid = domain, Grid(resolution)
        self.processes = [_DISCRETIZE[type(p)](p, domain, self.grid) for p in _flatten(processes)]
        fields = []
        for p in self.processes:                                        # state_fields (src/Processes.jl:77-87)
            names = ("vel1", "vel2", "vel3") if isinstance(
                p, (_DiscretizedAdvection, _DiscretizedSmagorinsky, _DiscretizedPressure)) else (p.field,)
            for f in names:
                if f not in fields:
                    fields.append(f)
        self.fields = [f for f in ("vel1", "vel2", "vel3") if f in fields]
        self.state = {f: self.zeros(f) for f in self.fields}
        self.transforms = {}
        self._t = self.transform(pdsize(self.grid))

    def zeros(self, field):
        g = self.grid
        return np.zeros((g.nz(NODES[field]), g.K2, g.K1), dtype=np.complex128)

    def transform(self, dims):
        dims = tuple(dims)
        if dims not in self.transforms:
            self.transforms[dims] = Transform2D(self.grid, dims)
        return self.transforms[dims]

    # -- hot path -------------------------------------------------------------------
    def compute_rates(self, state, rates=None, check=True):
        """compute_rates! + the finite check of rate! (src/Processes.jl:39-62, src/BoundaryLayerDynamics.jl:149-158)."""
        if rates is None:
            rates = {f: np.zeros_like(state[f]) for f in self.fields}
        else:
            for r in rates.values():
                r[...] = 0
        for p in self.processes:
            if p.kind == "linear":
                p.add_rates(rates, state)
        spaces = {}
        for p in self.processes:
            if p.kind == "nonlinear":
                dims = p.dims
                ps = spaces.setdefault(dims, {})
                for name in p.rate_names():
                    if name not in ps:
                        base = name.split("_")[0]
                        ps[name] = np.zeros((self.grid.nz(NODES[base]), dims[1], dims[0]))
                p.add_psrates(ps, state, self.transform(dims))
        D1 = dx1factors(self.domain, self.grid).reshape(1, -1)
        D2 = dx2factors(self.domain, self.grid).reshape(-1, 1)
        for dims, ps in spaces.items():                                 # add_rates! (src/physical_space.jl:191-204)
            tf = self.transform(dims)
            for name, values in ps.items():
                if "_" in name:
                    f, dd = name.split("_")
                    tf.add_field(rates[f], values, D1 if dd == "1" else D2)
                else:
                    tf.add_field(rates[name], values)
        if check:
            for r in rates.values():
                if not np.all(np.isfinite(r)):
                    raise DivergenceError("The simulation has diverged.")
        return rates

    def apply_projections(self, state):
        """apply_projections! (src/Processes.jl:67-75)."""
        for p in self.processes:
            if p.kind == "projection":
                p.apply_projection(state)
        return state

    # -- state I/O ------------------------------------------------------------------
    def coordinates(self, field, dims=None):
        dims = pdsize(self.grid) if dims is None else dims
        x1 = np.array([self.domain.hsize[0] * float(x) for x in h1range(dims[0])])
        x2 = np.array([self.domain.hsize[1] * float(x) for x in h1range(dims[1])])
        x3 = np.array([self.domain.vmap(z) for z in self.grid.vrange(NODES[field])])
        return x1, x2, x3

    def initialize(self, **ics):
        """initialize!(model; field = f) with f(x1, x2, x3) or an (n3, P2, P1) array (src/State.jl:11-31)."""
        for f in ics:
            if f not in self.state:
                raise KeyError(f"Cannot initialize `{f}`: unknown field")
        for f in self.fields:
            if f in ics:
                ic = ics[f]
                if callable(ic):
                    x1, x2, x3 = self.coordinates(f)
                    X3, X2, X1 = np.meshgrid(x3, x2, x1, indexing="ij")
                    vals = np.broadcast_to(np.asarray(ic(X1, X2, X3), dtype=np.float64), X1.shape)
                elif np.isscalar(ic):
                    x1, x2, x3 = self.coordinates(f)
                    vals = np.full((len(x3), len(x2), len(x1)), float(ic))
                else:
                    vals = np.asarray(ic, dtype=np.float64)
                self._t.set_field(self.state[f], np.ascontiguousarray(vals))
            else:
                self.state[f][...] = 0
        return self.state

    def __getitem__(self, field):
        """getterm at the default physical size (src/State.jl:81-85)."""
        return self._t.get_field(self.state[field])

    def get_field(self, field, dims=None, centered=False):
        t = self._t if dims is None else self.transform(dims)
        return t.get_field(self.state[field], centered=centered)

    def set_field(self, field, values, centered=False):
        """set_field! at the default size (src/physical_space.jl:253-256), e.g. from a snapshot."""
        self._t.set_field(self.state[field], np.ascontiguousarray(values, dtype=np.float64), centered=centered)

    # -- time integration -----------------------------------------------------------
    def rate(self):
        def rate_(du, u, t, checkpoint=False):
            st = dict(zip(self.fields, u))
            rt = dict(zip(self.fields, du))
            self.compute_rates(st, rt)
        return rate_

    def projection(self):
        def proj_(u):
            self.apply_projections(dict(zip(self.fields, u)))
        return proj_

    def evolve(self, tspan, dt, method=None):
        """evolve! (src/BoundaryLayerDynamics.jl:190-219)."""
        method = SSPRK33 if method is None else method
        t1, t2 = (0.0, float(tspan)) if np.isscalar(tspan) else (float(tspan[0]), float(tspan[1]))
        u0 = [self.state[f] for f in self.fields]
        prob = ODEProblem(self.rate(), self.projection(), u0, (t1, t2), checkpoint=True)
        if t2 > t1:
            nt = approxdiv(t2 - t1, dt)
            solve(prob, method, dt, checkpoints=list(np.linspace(t1 + dt, t2, nt)))
        return self


def approxdiv(a, b):                                                    # src/util.jl:19-24
    r = a / b
    ri = int(round(r))
    if not math.isclose(r, ri, rel_tol=math.sqrt(np.finfo(float).eps), abs_tol=0.0):
        raise ValueError("Division has a non-integer result")
    return ri


# --------------------------------------------------------------------------------------
# Explicit integrators (src/ODEMethods.jl)
# --------------------------------------------------------------------------------------

class ODEProblem:
    """``ODEProblem(rate!, projection!, u0, tspan)`` (src/ODEMethods.jl:168-185).

    ``u`` is a list of numpy arrays (the ArrayPartition); it is modified in place.
    """

    def __init__(self, rate, projection, u0, tspan, checkpoint=False):
        t1, t2 = tspan
        if t1 > t2:
            raise ValueError("Integration start time is larger than end time")
        self.rate_, self.projection_ = rate, (projection if projection is not None else (lambda u: None))
        self.u = u0
        self.du = [np.zeros_like(x) for x in u0]
        self.projection_(self.u)                                        # :182
        self._rate(self.du, self.u, t1, checkpoint=checkpoint)          # :183
        self.t, self.tmax = t1, t2

    def _rate(self, du, u, t, checkpoint=False):
        import inspect
        params = inspect.signature(self.rate_).parameters
        if "checkpoint" in params:
            self.rate_(du, u, t, checkpoint=checkpoint)
        else:
            self.rate_(du, u, t)


def _nanlike(u):
    return [np.full_like(x, np.nan) for x in u]


def Euler(prob):                                                        # :100-103
    def step(dt):
        for u, du in zip(prob.u, prob.du):
            u += dt * du
        prob.projection_(prob.u)
    return step


def AB2(prob):                                                          # :105-131
    state = {"duprev": _nanlike(prob.du), "last_dt": math.nan}

    def step(dt):
        if math.isnan(state["last_dt"]):
            for u, du in zip(prob.u, prob.du):
                u += dt * du
            prob.projection_(prob.u)
            for a, du in zip(state["duprev"], prob.du):
                a[...] = du
            prob._rate(prob.du, prob.u, prob.t + dt)
            for u, du, dp in zip(prob.u, prob.du, state["duprev"]):
                u += dt * (du - dp) / 2
            prob.projection_(prob.u)
            state["last_dt"] = dt
        else:
            if state["last_dt"] != dt:
                raise ValueError("Cannot change time step for multi-step methods")
            for u, du, dp in zip(prob.u, prob.du, state["duprev"]):
                u += dt / 2 * (3 * du - dp)
            prob.projection_(prob.u)
            for a, du in zip(state["duprev"], prob.du):
                a[...] = du
    return step


def SSPRK22(prob):                                                      # :133-145
    utmp = _nanlike(prob.u)

    def step(dt):
        for a, u, du in zip(utmp, prob.u, prob.du):
            a[...] = u + dt * du
        prob.projection_(utmp)
        prob._rate(prob.du, utmp, prob.t + dt)
        for u, a, du in zip(prob.u, utmp, prob.du):
            u[...] = (u + a + dt * du) / 2
        prob.projection_(prob.u)
    return step


def SSPRK33(prob):                                                      # :147-166
    utmp = _nanlike(prob.u)

    def step(dt):
        for a, u, du in zip(utmp, prob.u, prob.du):
            a[...] = u + dt * du
        prob.projection_(utmp)
        prob._rate(prob.du, utmp, prob.t + dt)
        for a, u, du in zip(utmp, prob.u, prob.du):
            a[...] = (3 * u + a + dt * du) / 4
        prob.projection_(utmp)
        prob._rate(prob.du, utmp, prob.t + dt / 2)
        for u, a, du in zip(prob.u, utmp, prob.du):
            u[...] = (u + 2 * a + 2 * dt * du) / 3
        prob.projection_(prob.u)
    return step


def solve(prob, alg, dt, checkpoints=None):
    """solve!/step_to! (src/ODEMethods.jl:198-234)."""
    step = alg(prob)
    if checkpoints is None or len(checkpoints) == 0:
        checkpoints = []
    elif min(checkpoints) <= prob.t or max(checkpoints) > prob.tmax:
        raise ValueError("Checkpoints outside of time range")
    else:
        checkpoints = sorted(checkpoints)
    for t in checkpoints:
        _step_to(prob, step, t, dt, True)
    _step_to(prob, step, prob.tmax, dt, False)
    return prob.u


def _isapprox(a, b):
    return a == b or abs(a - b) <= math.sqrt(np.finfo(float).eps) * max(abs(a), abs(b))


def _step_to(prob, step, t, dt, checkpoint):
    if _isapprox(prob.t, t):
        if checkpoint and prob.t != t:
            raise ValueError(f"Could not hit checkpoint t={t} exactly")
        prob.t = t
        return
    nt = approxdiv(t - prob.t, dt)
    for it in range(1, nt + 1):
        step(dt)
        prob.t = t if _isapprox(prob.t + dt, t) else prob.t + dt
        prob._rate(prob.du, prob.u, prob.t, checkpoint=(it == nt and checkpoint))
