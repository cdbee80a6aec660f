"""Laminar-flow integration tests of the reference, ported to pin the oracle's
time integration (test/laminar_test.jl, test/laminar_flow_problems.jl)."""

import math

import numpy as np
import pytest

from conftest import test_convergence

EPS = np.finfo(float).eps


def poiseuille(y, t, tol=EPS / 8, kmax=100_000):
    """test/laminar_flow_problems.jl:9-24"""
    if t == 0:
        return np.zeros_like(y)
    u = y - 0.5 * y ** 2
    if t == math.inf:
        return u
    for k in range(1, kmax + 1, 2):
        a = 16 / (k ** 3 * math.pi ** 3) * math.exp(-0.25 * k ** 2 * math.pi ** 2 * t)
        if a < tol:
            return u
        u = u - a * np.sin(0.5 * k * math.pi * y)
    return u


def couette(y, t, tol=EPS / 8, kmax=100_000):
    """test/laminar_flow_problems.jl:31-47"""
    if t == 0:
        return (y == 2).astype(float) - (y == 0).astype(float)
    u = np.zeros_like(y) + y - 1
    if t == math.inf:
        return u
    for k in range(1, kmax + 1):
        a = 2 / (k * math.pi) * math.exp(-k ** 2 * math.pi ** 2 * t)
        if a < tol:
            return u
        u = u + a * np.sin(y * k * math.pi)
    return u


def dx3_min(oracle, delta, N3, eta):
    """test/laminar_flow_problems.jl:57-62"""
    if eta is None:
        return 2 * delta / N3
    d = oracle.Domain((1, 1, 2 * delta), oracle.SmoothWall(), oracle.SmoothWall(), oracle.SinusoidalMapping(eta, "symmetric"))
    return min(d.Dvmap(z) for z in np.linspace(0, 1, 2 * N3 + 1)) / N3


def Nt_viscous(oracle, Nz, delta=1.0, nu=1.0, t=1.0, Cmax=0.5, eta=None):
    return math.ceil(t * nu / (Cmax * dx3_min(oracle, delta, Nz, eta) ** 2))


def _interp_vel3(field, lower=0.0, upper=0.0):
    """State.interpolate with Dirichlet vel3 (src/State.jl:87-99)."""
    ext = np.concatenate([np.full((1,) + field.shape[1:], lower), field, np.full((1,) + field.shape[1:], upper)])
    return (ext[:-1] + ext[1:]) / 2


def laminar_flow_error(oracle, Nh, Nv, Nt, u_exact, vel_bc=0.0, f=0.0, t=1.0, nu=1.0, delta=1.0, dir=(1.0, 0.0), eta=None, method=None):
    """test/laminar_flow_problems.jl:64-91"""
    nd = math.sqrt(dir[0] ** 2 + dir[1] ** 2)
    dir = (dir[0] / nd, dir[1] / nd)
    lbc = oracle.CustomBoundary(vel1=("dirichlet", -vel_bc * dir[0]), vel2=("dirichlet", -vel_bc * dir[1]), vel3="dirichlet")
    ubc = oracle.CustomBoundary(vel1=("dirichlet", vel_bc * dir[0]), vel2=("dirichlet", vel_bc * dir[1]), vel3="dirichlet")
    mapping = None if eta is None else oracle.SinusoidalMapping(eta, "symmetric")
    domain = oracle.Domain((1, 1, 2 * delta), lbc, ubc, mapping)
    model = oracle.Model((Nh, Nh, Nv), domain, oracle.incompressible_flow(nu, constant_forcing=(f * dir[0], f * dir[1])))
    model.evolve(t, t / Nt, method=method)
    x3 = model.coordinates("vel1")[2]
    uref = u_exact(x3, t).reshape(-1, 1, 1)
    e1 = model["vel1"] - uref * dir[0]
    e2 = model["vel2"] - uref * dir[1]
    e3 = _interp_vel3(model["vel3"])
    return math.sqrt(np.max(np.abs(e1) ** 2 + np.abs(e2) ** 2 + np.abs(e3) ** 2) / np.max(np.abs(uref) ** 2))


def taylor_green_vortex_error(oracle, Nh, Nv, Nt, t=1.0, nu=1.0, alpha=1.0, beta=1.0, gamma=1.0, U=1.0, W=None, eta=None, method=None):
    """test/laminar_flow_problems.jl:100-161"""
    tg1 = lambda x, y, t: np.sin(x) * np.cos(y) * np.exp(-t)
    tg2 = lambda x, y, t: -np.cos(x) * np.sin(y) * np.exp(-t)
    a, b, g = alpha, beta, gamma
    if W is None:
        refs = (lambda x, y, z, t: U * a * g * tg1(a * x + b * y, g * z, (a * a + b * b + g * g) * nu * t),
                lambda x, y, z, t: U * b * g * tg1(a * x + b * y, g * z, (a * a + b * b + g * g) * nu * t),
                lambda x, y, z, t: U * (a * a + b * b) * tg2(a * x + b * y, g * z, (a * a + b * b + g * g) * nu * t))
        bc = oracle.FreeSlipBoundary()
    else:
        refs = (lambda x, y, z, t: U * b * tg1(a * x, b * y, (a * a + b * b) * nu * t),
                lambda x, y, z, t: U * a * tg2(a * x, b * y, (a * a + b * b) * nu * t),
                lambda x, y, z, t: W + 0 * x)
        bc = oracle.CustomBoundary(vel1="neumann", vel2="neumann", vel3=("dirichlet", W))
    ds = (2 * math.pi / a, 2 * math.pi / b, 2 * math.pi / g)
    mapping = None if eta is None else oracle.SinusoidalMapping(eta, "symmetric")
    domain = oracle.Domain(ds, bc, bc, mapping)
    model = oracle.Model((Nh, Nh, Nv), domain, oracle.incompressible_flow(nu, constant_forcing=0))
    model.initialize(**{f: (lambda r: (lambda x, y, z: r(x, y, z, 0.0)))(r) for f, r in zip(("vel1", "vel2", "vel3"), refs)})
    model.evolve(t, t / Nt, method=method)
    errs = []
    for f, r in zip(("vel1", "vel2", "vel3"), refs):
        x1, x2, x3 = model.coordinates(f)
        X3, X2, X1 = np.meshgrid(x3, x2, x1, indexing="ij")
        errs.append(model[f] - r(X1, X2, X3, t))
    w = 0.0 if W is None else W
    e3 = _interp_vel3(errs[2], 0.0 * w, 0.0 * w)
    uref_max = math.exp(-nu * t * (a * a + b * b + (g * g if W is None else 0)))
    return math.sqrt(np.max(np.abs(errs[0]) ** 2 + np.abs(errs[1]) ** 2 + np.abs(e3) ** 2) / uref_max)


@pytest.mark.parametrize("grid_stretching", [False, True])
def test_laminar_flow_convergence(oracle, grid_stretching):
    """test/laminar_test.jl:3-65 (Poiseuille, Couette, Taylor-Green; spatial and temporal orders)."""
    rng = np.random.default_rng(62275)
    Nz_min = 3
    N = [n for n in (11, 14, 18, 24) if n >= Nz_min]
    eta = 0.4 + rng.random() / 5 if grid_stretching else None
    nu = 3 / 4 + rng.random() / 2
    th = rng.random() * 2 * math.pi
    ex = (math.cos(th), math.sin(th))
    delta = 3 / 4 + rng.random() / 2
    utau = 3 / 4 + rng.random() / 2
    t = (delta ** 2 / nu) / 6
    Nt = Nt_viscous(oracle, N[-1], delta=delta, nu=nu, t=t, Cmax=0.25, eta=eta)
    m = oracle.SSPRK22
    ep = [laminar_flow_error(oracle, 3, n, Nt, lambda y, tt: (utau ** 2 * delta / nu) * poiseuille(y / delta, tt * nu / delta ** 2),
                             f=utau ** 2 / delta, t=t, nu=nu, delta=delta, dir=ex, eta=eta, method=m) for n in N]
    ec = [laminar_flow_error(oracle, 3, n, Nt, lambda y, tt: (utau ** 2 * delta / nu) * couette(y / delta, tt * nu / delta ** 2),
                             vel_bc=utau * utau * delta / nu, t=t, nu=nu, delta=delta, dir=ex, eta=eta, method=m) for n in N]
    a, b, g, U = (3 / 4 + rng.random() / 2 for _ in range(4))
    t = 1 / ((a * a + b * b + g * g) * nu)
    Nt = Nt_viscous(oracle, N[-1], delta=math.pi / (2 * b), nu=nu, t=t, Cmax=0.25)
    kw = dict(t=t, nu=nu, alpha=a, beta=b, gamma=g, U=U, eta=eta)
    etgv = [taylor_green_vortex_error(oracle, 3, n, Nt, method=m, **kw) for n in N]
    kw["W"] = 0.0
    eeu = [taylor_green_vortex_error(oracle, 3, Nz_min, n, method=oracle.Euler, **kw) for n in N]
    eab = [taylor_green_vortex_error(oracle, 3, Nz_min, n, method=oracle.AB2, **kw) for n in N]
    er2 = [taylor_green_vortex_error(oracle, 3, Nz_min, n, method=oracle.SSPRK22, **kw) for n in N]
    er3 = [taylor_green_vortex_error(oracle, 3, Nz_min, n, method=oracle.SSPRK33, **kw) for n in N]
    assert ep[-1] < (1e-3 if grid_stretching else 2e-3)
    assert ec[-1] < (1e-3 if grid_stretching else 5e-4)
    assert etgv[-1] < (7e-3 if grid_stretching else 5e-3)
    test_convergence(N, ep, order=2, threshold_slope=0.95)
    test_convergence(N, ec, order=2, threshold_slope=0.9)
    test_convergence(N, etgv, order=2, threshold_slope=0.94)
    assert eeu[-1] < 2e-2 and eab[-1] < 4e-4 and er2[-1] < 2e-4 and er3[-1] < 2e-6
    test_convergence(N, eeu, order=1, threshold_slope=0.99)
    test_convergence(N, eab, order=2, threshold_slope=0.98)
    test_convergence(N, er2, order=2, threshold_slope=0.99)
    test_convergence(N, er3, order=3, threshold_slope=0.99)


def test_constant_flux_poiseuille(oracle):
    """test/laminar_test.jl:67-100: constant flux converges faster than constant forcing."""
    nz = 16
    z = np.linspace(0, 2, 2 * nz + 1)[1::2]
    u_exact = poiseuille(z, math.inf)
    mf = np.sum(u_exact) / nz
    CFL, nu, tend, nit = (1 / 4, 1.0, 1.0, 8)
    dtmax = (2 / nz) ** 2 / nu * CFL
    nt = math.ceil(tend / dtmax / nit)
    dt = tend / (nit * nt)
    domain = oracle.Domain((4 * math.pi, 2 * math.pi, 2), oracle.SmoothWall(), oracle.SmoothWall())
    m1 = oracle.Model((4, 4, nz), domain, oracle.incompressible_flow(1.0, constant_forcing=1))
    m2 = oracle.Model((4, 4, nz), domain, oracle.incompressible_flow(1.0, constant_flux=mf))
    eps = lambda m: np.sum(np.abs(m.state["vel1"][:, 0, 0] - u_exact)) / nz
    ef, eq = [], []
    for _ in range(nit):
        m1.evolve(dt * nt, dt)
        ef.append(eps(m1))
        m2.evolve(dt * nt, dt)
        eq.append(eps(m2))
    assert all(q < f for q, f in zip(eq, ef))
    assert all(np.diff(eq) < 0)
    assert eq[-1] < 1e-6
