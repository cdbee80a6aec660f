"""Output modules for ``evolve`` (src/logging.jl): Snapshots, MeanProfiles and
ProgressMonitor.

Both work on the device-resident state.  ``Snapshots`` reads the physical fields
back only at its output times (centered transforms run on the device) and
writes one CBD file per field, in the reference's folder layout
``<path>/state-NNN/<field>.cbd``.  ``MeanProfiles`` lets the step graphs
integrate the horizontal means on the device after every step (trapezoidal rule
in time, as the reference samples at every checkpoint) and reads back only the
integrals, 3 (n3 + 1) numbers, at its output times.  The reference writes the
profiles to HDF5 (``<path>-NN.h5``); h5py is not part of this stack, so the same
datasets (the profiles, ``intervals``, ``timespan``) go to ``<path>-NN.npz``.
"""

import math
import os
from fractions import Fraction

import numpy as np

from . import cbd


def _multiple(t, freq):
    """t / freq is (approximately) an integer n >= 1 (log_state!, src/logging.jl:586-588)."""
    if t == 0:
        return None
    n = round(t / freq)
    return n if n >= 1 and math.isclose(n, t / freq, rel_tol=1e-9) else None


class Snapshots:
    """``Snapshots(frequency=..., path="output/snapshots", centered=True, precision=np.float64)``
    (src/logging.jl:527-601)."""

    def __init__(self, frequency, path=os.path.join("output", "snapshots"), centered=True, precision=np.float64):
        if frequency is None or frequency <= 0:
            raise ValueError("Snapshots need a positive frequency")
        self.frequency = float(frequency)
        self.path = path
        self.centered = bool(centered)
        self.precision = np.dtype(precision)
        self.written = []

    def output_times(self, t1, t2):
        n1 = math.floor(t1 / self.frequency + 1e-9) + 1
        n2 = math.floor(t2 / self.frequency + 1e-9)
        return [n * self.frequency for n in range(n1, n2 + 1)]

    def start(self, model, t):
        self.model = model

    def at(self, model, t, steps=0, member=0):
        n = _multiple(t, self.frequency)
        if n is None:
            return
        folder = os.path.join(self.path, "state-%03d" % n)
        xmin, xmax = snapshot_limits(model)
        for field in model.fields:
            x1, x2, x3 = snapshot_coordinates(model, field, self.centered)
            values = model.get_field(field, member=member, centered=self.centered)
            fn = os.path.join(folder, f"{field}.cbd")
            cbd.writecbd(self.precision, fn, values, x1, x2, x3, xmin, xmax)
            self.written.append(fn)

    def finish(self, model, t):
        pass


class MeanProfiles:
    """``MeanProfiles(profiles=("vel1", "vel2", "vel3"), path="output/profiles", output_frequency=...)``
    (src/logging.jl:333-491), integrated on the device."""

    def __init__(self, profiles=("vel1", "vel2", "vel3"), path=os.path.join("output", "profiles"),
                 output_frequency=None):
        for p in profiles:
            if p not in ("vel1", "vel2", "vel3"):
                raise ValueError(f"profiles of `{p}` are not collected on the device")
        self.profiles = tuple(profiles)
        self.path = path
        self.output_frequency = output_frequency
        self.files = []
        self.last = None

    def output_times(self, t1, t2):
        if not self.output_frequency:
            return []
        f = float(self.output_frequency)
        n1 = math.floor(t1 / f + 1e-9) + 1
        n2 = math.floor(t2 / f + 1e-9)
        return [n * f for n in range(n1, n2 + 1)]

    def start(self, model, t):
        self.model = model
        self.timespan = [t, t]
        self.intervals = 0
        model.profiles_start(True)

    def _read(self, model, member=0):
        raw = model.profiles_read(member)
        n3 = model.n3
        out = {}
        for i, f in enumerate(("vel1", "vel2", "vel3")):
            row = raw[i * (n3 + 1):(i + 1) * (n3 + 1)]
            if f in self.profiles:
                out[f] = row.copy() if f == "vel3" else row[:n3].copy()
        return out

    def at(self, model, t, steps):
        """Called at an output time after ``steps`` steps since the last call."""
        self.intervals += steps
        self.timespan[1] = t
        if self.output_frequency and _multiple(t, float(self.output_frequency)) is not None:
            self.flush(model)

    def flush(self, model, member=0):
        """flush! (src/logging.jl:453-491): time averages over the interval, written to the next free file."""
        if self.intervals == 0:
            return None
        dt = self.timespan[1] - self.timespan[0]
        if not dt > 0:
            raise ValueError("Time interval for averaging is not positive")
        means = {f: v / dt for f, v in self._read(model, member).items()}
        folder, prefix = os.path.dirname(self.path), os.path.basename(self.path) + "-"
        if folder:
            os.makedirs(folder, exist_ok=True)
        i = 1
        while os.path.exists(os.path.join(folder, prefix + "%02d.npz" % i)):
            i += 1
        fn = os.path.join(folder, prefix + "%02d.npz" % i)
        np.savez(fn, intervals=self.intervals, timespan=np.array(self.timespan), **means)
        self.files.append(fn)
        self.last = means
        # reset! (:493-500): the next interval starts here, with the current state as first sample
        self.intervals = 0
        self.timespan[0] = self.timespan[1]
        model.profiles_start(True)
        return fn

    def finish(self, model, t):
        self.flush(model)
        model.profiles_start(False)


def snapshot_limits(model):
    """extrema(domain) (src/Domains.jl): ((0, 0, x3min), (L1, L2, x3max))."""
    L1, L2 = model.domain.hsize
    x3min, x3max = model.domain.extrema3()
    return (0.0, 0.0, float(x3min)), (float(L1), float(L2), float(x3max))


def snapshot_coordinates(model, field, centered):
    """x1range/x2range of h1range/h2range(default size; centered) and x3 of the field's nodes
    (src/physical_space.jl:64-65, src/logging.jl:565-570)."""
    P1, P2 = model.default_size
    L1, L2 = model.domain.hsize
    c = 1 if centered else 0
    x1 = np.array([L1 * float(Fraction(2 * i + c, 2 * P1)) for i in range(P1)])
    x2 = np.array([L2 * float(Fraction(2 * i + c, 2 * P2)) for i in range(P2)])
    return x1, x2, model.coordinates(field)[2]


def initialize_from_snapshot(model, path, member=0):
    """initialize!(model, path) (src/State.jl:33-66): fields from ``<path>/<field>.cbd``,
    zero (with a warning) where a file is missing."""
    import warnings
    xmin, xmax = snapshot_limits(model)
    P1, P2 = model.default_size
    for field in model.fields:
        fn = os.path.join(path, f"{field}.cbd")
        if not os.path.isfile(fn):
            warnings.warn(f"No initial values found for `{field}`, set to zero.")
            model.set_field(field, 0.0, member=member)
            continue
        fxmin, fxmax, x1, x2, x3, data = cbd.readcbd(fn, model.coordinates(field)[2])
        if not (np.allclose(fxmin, xmin) and np.allclose(fxmax, xmax)):
            raise ValueError(f"{fn}: domain limits do not match the model")
        centered = x1[0] != 0
        if data.shape[1:] != (P2, P1):
            raise ValueError(f"{fn}: snapshot size {data.shape[1:][::-1]} differs from the default size {(P1, P2)}")
        ex1, ex2, ex3 = snapshot_coordinates(model, field, centered)
        if not (np.allclose(x1, ex1) and np.allclose(x2, ex2) and np.allclose(x3, ex3)):
            raise ValueError(f"{fn}: coordinates do not match the model")
        model.set_field(field, np.asarray(data, dtype=np.float64), member=member, centered=centered)


class ProgressMonitor:
    """``ProgressMonitor(frequency=10, description="Progress:", tstep=None)``
    (src/logging.jl:129-308): prints the progress and the flow statistics at
    intervals of wall time.  The statistics come from the device-resident state
    (``Model.progress``: mean velocity, mean and turbulent kinetic energy, the
    advective time scale or Courant number, wall stresses); the state is checked
    every ``check_every`` steps (the reference checks after every step, which
    would break the multi-step device launches), and always at the end."""

    def __init__(self, frequency=10, description="Progress:", tstep=None, checks=20, stream=None):
        import sys
        self.frequency = float(frequency)
        self.description = description
        self.tstep = tstep
        self.checks = int(checks)   # times the run is split for the wall-time checks
        self.stream = stream or sys.stdout
        self.reports = []      # (simulation time, statistics) of every report
        self._dt = None

    def set_dt(self, dt):
        self._dt = float(dt)

    def output_times(self, t1, t2):
        self._t1, self._t2 = t1, t2
        if not self._dt or self.checks < 2:
            return []
        n = int(round((t2 - t1) / self._dt))
        every = max(1, n // self.checks)
        return [t1 + k * self._dt for k in range(every, n, every)]

    def start(self, model, t):
        import time
        self._start = time.time()
        self._last = None

    def at(self, model, t, steps=0, member=0):
        import time
        now = time.time()
        progress = (t - self._t1) / (self._t2 - self._t1) if self._t2 > self._t1 else 1.0
        if self._last is not None and now - self._last < self.frequency and progress < 1:
            return
        self._last = now
        stats = {"Simulation Time": t}
        stats.update(model.progress(member=member, tstep=self.tstep))
        self.reports.append((t, stats))
        rate = progress / max(now - self._start, 1e-9)
        eta = (1 - progress) / rate if rate > 0 else float("inf")
        print(f"{self.description} {100 * progress:3.0f}%  ETA: {eta:.0f} s", file=self.stream)
        width = max(len(k) for k in stats) + 2
        for k, v in stats.items():
            vals = ", ".join(f"{x:.3g}" for x in (v if isinstance(v, tuple) else (v,)))
            print(f"{k:>{width}} ╎ {vals}", file=self.stream)

    def finish(self, model, t):
        if not self.reports or self.reports[-1][0] != t:
            self._last = None
            self.at(model, t)
