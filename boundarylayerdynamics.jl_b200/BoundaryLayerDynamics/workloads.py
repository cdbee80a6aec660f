"""Seeded synthetic workloads: the five benchmark configurations as plain specs.

A spec is library-agnostic: ``build(spec, api)`` instantiates it with any
module that exposes the reference's constructor names (``Domain``,
``RoughWall``, ``incompressible_flow``, ``StaticSmagorinskyModel``,
``Model`` ...), and ``initial_fields(spec, ...)`` returns the seeded
physical-space initial condition on the default grid, so every consumer sees
identical input values.

Choices the benchmark description leaves open (recorded here, once):
* half-channel LES: nu = 1e-5, u* = 1, kappa = 0.4;
* closed-channel DNS: centreline velocity U_c = 18, dt = 1e-4.
"""

import math

import numpy as np

LES_Z0 = 1e-4
KAPPA = 0.4
DNS_UC = 18.0


def les_spec(n, nz, size, seed=0, z0=LES_Z0, cs=0.1, forcing=1.0, dt=1e-4, steps=100, nu=1e-5):
    return dict(kind="les", resolution=(n, n, nz), size=size, lower=("rough", z0), upper=("freeslip",),
                nu=nu, forcing=forcing, sgs=dict(Cs=cs), dt=dt, steps=steps, seed=seed)


def dns_spec(n, nz, seed=0, dt=1e-4, steps=1000, Re=180.0):
    return dict(kind="dns", resolution=(n, n, nz), size=(4 * math.pi, 2 * math.pi, 2.0), lower=("smooth",),
                upper=("smooth",), nu=1.0 / Re, forcing=1.0, sgs=None, dt=dt, steps=steps, seed=seed)


CONFIGS = {
    # Plain LES of a half-channel ABL, 64x64x32 on 2pi x pi x 1, SSPRK33, dt=1e-4, 100 steps
    "les64": les_spec(64, 32, (2 * math.pi, math.pi, 1.0)),
    # DNS of a closed channel, 192x192x96 on 4pi x 2pi x 2, nu = 1/180, 1000 steps
    "dns192": dns_spec(192, 96),
    # Large LES, 512x512x256 on 8pi x 4pi x 1
    "les512": les_spec(512, 256, (8 * math.pi, 4 * math.pi, 1.0)),
}


def _wall(api, w):
    if w[0] == "rough":
        return api.RoughWall(w[1])
    if w[0] == "smooth":
        return api.SmoothWall()
    if w[0] == "freeslip":
        return api.FreeSlipBoundary()
    raise ValueError(w)


def build(spec, api, **model_kw):
    """Instantiate ``spec`` with the constructors of ``api``; returns the Model."""
    domain = api.Domain(spec["size"], _wall(api, spec["lower"]), _wall(api, spec["upper"]))
    sgs = api.StaticSmagorinskyModel(Cs=spec["sgs"]["Cs"]) if spec.get("sgs") else None
    procs = api.incompressible_flow(spec["nu"], constant_forcing=spec["forcing"], sgs_model=sgs)
    return api.Model(spec["resolution"], domain, procs, **model_kw)


def default_grid(spec):
    """x1, x2 of the default physical grid and x3 of the C and I nodes."""
    n1, n2, n3 = spec["resolution"]
    P1, P2 = 2 * ((n1 - 1) // 2) + 2, 2 * ((n2 - 1) // 2) + 2
    L1, L2, L3 = spec["size"]
    x1 = L1 * np.arange(P1) / P1
    x2 = L2 * np.arange(P2) / P2
    x3c = L3 * (2 * np.arange(1, n3 + 1) - 1) / (2 * n3)
    x3i = L3 * np.arange(1, n3) / n3
    return x1, x2, x3c, x3i


def initial_fields(spec, seed=None):
    """Seeded physical-space initial condition (u, v, w) on the default grid.

    LES: u = (u*/kappa) ln(z/z0) (1 + r), v and w = (u*/kappa) ln(z/z0) r with r ~ U(-0.1, 0.1).
    DNS: u = U_c (1 - (z-1)^2) + n, v = n, w = n with n ~ N(0, (0.05 U_c)^2).
    """
    seed = spec["seed"] if seed is None else seed
    rng = np.random.default_rng(seed)
    x1, x2, x3c, x3i = default_grid(spec)
    P1, P2 = len(x1), len(x2)
    nc, ni = len(x3c), len(x3i)
    if spec["kind"] == "les":
        z0 = spec["lower"][1]
        prof_c = (np.log(x3c / z0) / KAPPA)[:, None, None]
        prof_i = (np.log(x3i / z0) / KAPPA)[:, None, None]
        r = lambda n: rng.uniform(-0.1, 0.1, size=(n, P2, P1))
        u = prof_c * (1 + r(nc))
        v = prof_c * r(nc)
        w = prof_i * r(ni)
    else:
        sig = 0.05 * DNS_UC
        u = (DNS_UC * (1 - (x3c - 1) ** 2))[:, None, None] + rng.normal(0, sig, size=(nc, P2, P1))
        v = rng.normal(0, sig, size=(nc, P2, P1))
        w = rng.normal(0, sig, size=(ni, P2, P1))
    return u, v, w


# ----------------------------------------------------------- seeded fields on the device
_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(x):
    """SplitMix64's output function (Steele, Lea and Flood, OOPSLA 2014) of uint64 x,
    elementwise, with 64-bit wraparound: the generator of bld_init_random_field."""
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + _GAMMA
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def seeded_field(shape, base, scale, distribution, seed, field):
    """The values bld_init_random_field puts on the default grid: base[z] + scale[z] r
    with r uniform on [-1, 1) or standard normal, counter i = (z P2 + y) P1 + x."""
    nz, P2, P1 = shape
    with np.errstate(over="ignore"):
        key = splitmix64(np.uint64(seed)) ^ splitmix64(np.uint64(field + 1))
        i = np.arange(nz * P2 * P1, dtype=np.uint64)
        u = (splitmix64(key + np.uint64(2) * i) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
        if distribution == "uniform":
            r = 2.0 * u - 1.0
        else:
            u2 = (splitmix64(key + np.uint64(2) * i + np.uint64(1)) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
            r = np.sqrt(-2.0 * np.log(1.0 - u)) * np.cos(2.0 * np.pi * u2)
    r = r.reshape(nz, P2, P1)
    return np.asarray(base, float)[:, None, None] + np.asarray(scale, float)[:, None, None] * r


def seeded_profiles(spec):
    """(base, scale, distribution) per field of the workload's initial condition in
    the form the device generator takes: LES u = p (1 + 0.1 r), v = 0.1 p r,
    w = 0.1 p_I r with p = (u*/kappa) ln(z/z0) and r uniform on [-1, 1); DNS
    u = U_c (1 - (z - 1)^2) + sigma n, v = sigma n, w = sigma n with
    sigma = 0.05 U_c and n standard normal."""
    _, _, x3c, x3i = default_grid(spec)
    if spec["kind"] == "les":
        z0 = spec["lower"][1]
        pc, pi = np.log(x3c / z0) / KAPPA, np.log(x3i / z0) / KAPPA
        return {"vel1": (pc, 0.1 * pc, "uniform"), "vel2": (0 * pc, 0.1 * pc, "uniform"),
                "vel3": (0 * pi, 0.1 * pi, "uniform")}
    sig = 0.05 * DNS_UC
    return {"vel1": (DNS_UC * (1 - (x3c - 1) ** 2), sig + 0 * x3c, "normal"),
            "vel2": (0 * x3c, sig + 0 * x3c, "normal"), "vel3": (0 * x3i, sig + 0 * x3i, "normal")}


def seeded_initial_fields(spec, seed):
    """Host copies of the fields initialize_on_device builds (u, v, w on the default grid)."""
    x1, x2, x3c, x3i = default_grid(spec)
    P1, P2 = len(x1), len(x2)
    out = []
    for k, (f, (b, sc, dist)) in enumerate(seeded_profiles(spec).items()):
        nz = len(x3c) if f != "vel3" else len(x3i)
        out.append(seeded_field((nz, P2, P1), b, sc, dist, seed, k))
    return tuple(out)


def initialize_on_device(spec, model, seed, member=0):
    """initialize! with the workload's seeded initial condition generated on the device."""
    for f, (b, sc, dist) in seeded_profiles(spec).items():
        model.init_random_field(f, b, sc, dist, seed, member)


def ensemble_members(seed=3):
    """The 64-member uneven ensemble: 24 x 64^2x32, 24 x 96^2x48, 16 x 128^2x64 with
    z0 ~ logU[1e-5, 1e-3] and Cs ~ U[0.08, 0.16] per member."""
    rng = np.random.default_rng(seed)
    groups = []
    for n, nz, count in ((64, 32, 24), (96, 48, 24), (128, 64, 16)):
        z0 = np.exp(rng.uniform(math.log(1e-5), math.log(1e-3), size=count))
        cs = rng.uniform(0.08, 0.16, size=count)
        groups.append(dict(spec=les_spec(n, nz, (2 * math.pi, math.pi, 1.0)), z0=z0, cs=cs))
    return groups
