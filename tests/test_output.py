"""Output formats on the CPU: CBD files and the half-grid-point shift.

Known-answer tests restated from the reference's test/output_test.jl:
test_file_io (a linear field through set_field!/get_field and a CBD round trip,
in both precisions and for C and I nodes) and test_shifted_file_output (the
centered transform reproduces an analytic field at the interval centres).  The
package's CBD writer must produce the same bytes as the oracle's.
"""

import math
import os

import numpy as np
import pytest

from BoundaryLayerDynamics import cbd


def _grid_model(oracle, n1, n2, n3, ds):
    dom = oracle.Domain(ds, oracle.FreeSlipBoundary(), oracle.FreeSlipBoundary())
    return oracle.Model((n1, n2, n3), dom, [oracle.MolecularDiffusion("vel1", 1.0),
                                            oracle.MolecularDiffusion("vel3", 1.0)])


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("ns", ["C", "I"])
def test_file_io(oracle, tmp_path, T, ns):
    """test/output_test.jl:1-44: x/L1 + y/L2 + z/L3 written and read back."""
    rng = np.random.default_rng(73330459108 % 2**32)
    n1, n2, n3 = 6, 8, 12
    ds = tuple(float(T(v)) for v in rng.random(3) + 0.5)
    om = _grid_model(oracle, n1, n2, n3, ds)
    field = "vel1" if ns == "C" else "vel3"
    om.initialize(**{field: lambda x, y, z: x / ds[0] + y / ds[1] + z / ds[2]})
    vel = om.get_field(field)
    P2, P1 = vel.shape[1:]
    x1 = np.linspace(0, ds[0], P1 + 1)[:P1]
    x2 = np.linspace(0, ds[1], P2 + 1)[:P2]
    x3 = np.linspace(0, ds[2], 2 * n3 + 1)[(1 if ns == "C" else 2):-1:2]
    xmin, xmax = (0.0, 0.0, 0.0), ds
    for Tf in (np.float32, np.float64):
        fn = str(tmp_path / f"vel-{np.dtype(Tf).name}-{ns}.cbd")
        cbd.writecbd(Tf, fn, vel, x1, x2, x3, xmin, xmax)
        xmin_a, xmax_a, x1_a, x2_a, x3_a, vel_a = cbd.readcbd(fn, x3)
        assert xmin_a == xmin and tuple(xmax_a) == tuple(ds)
        assert np.array_equal(x1_a, x1) and np.array_equal(x2_a, x2) and np.array_equal(x3_a, x3)
        if Tf == np.float64:
            assert np.array_equal(vel_a, vel)
        else:
            assert np.allclose(vel_a, vel, rtol=1e-6, atol=1e-6)


def test_cbd_bytes_match_oracle(oracle, tmp_path):
    rng = np.random.default_rng(1)
    field = rng.standard_normal((5, 4, 6))
    x1, x2, x3 = np.arange(6) * 0.5, np.arange(4) * 0.25, np.linspace(0.1, 0.9, 5)
    for T in (np.float32, np.float64):
        a, b = str(tmp_path / "a.cbd"), str(tmp_path / "b.cbd")
        cbd.writecbd(T, a, field, x1, x2, x3, (0, 0, 0), (3, 1, 1))
        oracle.writecbd(T, b, field, x1, x2, x3, (0, 0, 0), (3, 1, 1))
        with open(a, "rb") as fa, open(b, "rb") as fb:
            ba, bb = fa.read(), fb.read()
        assert ba == bb
        assert ba[:3] == bytes([0xCB, 0xDF, 1]) and ba[7] == np.dtype(T).itemsize
        assert len(ba) == 8 + 24 + 48 + 8 * (6 + 4 + 5) + np.dtype(T).itemsize * field.size


def test_cbd_x3_range(tmp_path):
    """readcbd returns the layers covering the requested x3 interval (src/fileio.jl:93-101)."""
    field = np.arange(7 * 2 * 3, dtype=float).reshape(7, 2, 3)
    x3 = np.linspace(0, 1, 7)
    fn = str(tmp_path / "r.cbd")
    cbd.writecbd(np.float64, fn, field, [0, 1, 2], [0, 1], x3, (0, 0, 0), (1, 1, 1))
    _, _, _, _, x3r, data = cbd.readcbd(fn, (x3[2], x3[4]))
    assert np.array_equal(x3r, x3[2:5]) and np.array_equal(data, field[2:5])
    with pytest.raises(ValueError, match="magic"):
        with open(fn, "r+b") as f:
            f.write(b"XX")
        cbd.readcbd(fn)


@pytest.mark.parametrize("ns", ["C", "I"])
def test_shifted_file_output(oracle, tmp_path, ns):
    """test/output_test.jl:46-91: the centered transform reproduces the analytic field
    at the centres of the grid intervals."""
    rng = np.random.default_rng(839905175168 % 2**32)
    n1, n2, n3 = 6, 8, 12
    k1max, k2max = (n1 - 1) // 2, (n2 - 1) // 2
    C0, Cx, Cy = rng.random(), rng.random((2, k1max)), rng.random((2, k2max))

    def vel0(x, y, z):
        sx = sum(Cx[0, i] * np.sin((i + 1) * x + Cx[1, i]) for i in range(k1max))
        sy = sum(Cy[0, i] * np.sin((i + 1) * y + Cy[1, i]) for i in range(k1max))
        return (sx + sy + C0) * z * (1 - z)

    ds = (2 * math.pi, 2 * math.pi, 1.0)
    om = _grid_model(oracle, n1, n2, n3, ds)
    field = "vel1" if ns == "C" else "vel3"
    om.initialize(**{field: vel0})
    vel = om.get_field(field, centered=True)
    P2, P1 = vel.shape[1:]
    x1 = np.linspace(0, ds[0], 2 * P1 + 1)[1:-1:2]
    x2 = np.linspace(0, ds[1], 2 * P2 + 1)[1:-1:2]
    x3 = np.linspace(0, ds[2], 2 * n3 + 1)[1:-1][(0 if ns == "C" else 1)::2]
    fn = str(tmp_path / f"vel-{ns}.cbd")
    cbd.writecbd(np.float64, fn, vel, x1, x2, x3, (0, 0, 0), ds)
    _, _, x1f, x2f, x3f, data = cbd.readcbd(fn, x3)
    X3, X2, X1 = np.meshgrid(x3f, x2f, x1f, indexing="ij")
    assert np.allclose(data, vel0(X1, X2, X3), rtol=1e-12, atol=1e-12)


def test_centered_round_trip_oracle(oracle):
    """set_field!(...; centered) inverts get_field(...; centered) on resolved modes."""
    om = _grid_model(oracle, 12, 10, 5, (1.0, 2.0, 1.0))
    rng = np.random.default_rng(4)
    st = om.state["vel1"]
    st[...] = rng.standard_normal(st.shape) + 1j * rng.standard_normal(st.shape)
    st[:, 0, 0] = st[:, 0, 0].real
    pd = om.get_field("vel1", centered=True)
    before = st.copy()
    om.set_field("vel1", pd, centered=True)
    # modes that survive a real round trip (k1 = 0 keeps only its Hermitian part)
    assert np.allclose(om.state["vel1"][:, :, 1:], before[:, :, 1:], atol=1e-12)


def test_mean_profiles_oracle_trapezoid(oracle):
    """A steady state gives its own mean profile (the trapezoidal weights sum to the span)."""
    mp = oracle.MeanProfiles(4, 0.0)
    st = {"vel1": np.zeros((4, 3, 2), complex), "vel2": np.zeros((4, 3, 2), complex),
          "vel3": np.zeros((3, 3, 2), complex)}
    st["vel1"][:, 0, 0] = [1, 2, 3, 4]
    st["vel3"][:, 0, 0] = [5, 6, 7]
    mp.sample_state(st)
    for k in range(1, 6):
        mp.step(st, 0.1 * k)
    avg = mp.averages()
    assert np.allclose(avg["vel1"], [1, 2, 3, 4]) and np.allclose(avg["vel3"], [0, 5, 6, 7, 0])
    assert mp.intervals == 5


def test_progress_monitor_checks_and_reports():
    """ProgressMonitor's host logic with a fake model: the check times fall on
    whole steps, reports follow the wall-time interval and the last one comes
    at the end time (src/logging.jl:175-191)."""
    import io
    import BoundaryLayerDynamics.output as out

    class Fake:
        def progress(self, member=0, tstep=None):
            return {"Mean Velocity": (1.0, 0.0, 0.0), "Mean KE": 0.5, "Turbulent KE": 0.1,
                    "Adv. Courant Number": 0.2}

    buf = io.StringIO()
    pm = out.ProgressMonitor(frequency=1e9, tstep=0.1, checks=5, stream=buf)
    pm.set_dt(0.1)
    times = pm.output_times(0.0, 2.0)
    assert times == pytest.approx([0.4, 0.8, 1.2, 1.6])
    model = Fake()
    pm.start(model, 0.0)
    for t in times:
        pm.at(model, t)
    pm.finish(model, 2.0)
    # the first check reports, the others fall inside the (huge) wall-time interval,
    # the end always reports
    assert [t for t, _ in pm.reports] == pytest.approx([0.4, 2.0])
    assert "Turbulent KE" in buf.getvalue()
