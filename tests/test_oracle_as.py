"""The axisymmetric oracle (kspaceFirstOrderAS.m, radial symmetry 'WSWA-FFT').

Pins: the radial mirror has the reference's symmetry; a field that is
rotationally symmetric about an axis, run on the axisymmetric grid, matches
the same field run in 3D with that axis through grid points (two different
discretisations of one physical problem, so to a percent); the front end
builds the axisymmetric datasets."""
import numpy as np
import pytest

from oracle.kspace_oracle import simulate
from oracle.kspace_oracle_as import mirror_p, mirror_sg, simulate_as


def test_mirror_symmetries():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((3, 6))
    m = mirror_p(a, 6)
    # even about the axis (index 0, period 24) and odd about the outer radius (index 6)
    for j in range(1, 6):
        np.testing.assert_array_equal(m[:, -j], m[:, j])
        np.testing.assert_array_equal(m[:, 6 + j], -m[:, 6 - j])
    assert not m[:, 6].any() and not m[:, 18].any()
    s = mirror_sg(a, 6)  # staggered points: (j + 1/2) dy
    for j in range(6):
        np.testing.assert_array_equal(s[:, 23 - j], -s[:, j])   # odd about the axis
        np.testing.assert_array_equal(s[:, 6 + j], s[:, 5 - j])  # even about the outer radius


def _ball_inputs(nx, ny, nt, dx, c, center_x):
    xx = np.arange(nx)[:, None] - center_x
    yy = np.arange(ny)[None, :]
    p0 = np.exp(-(xx.astype(float) ** 2 + yy ** 2) / 6.0)
    return dict(Nx=nx, Ny=ny, Nz=1, Nt=nt, dx=dx, dy=dx, dz=0.0, dt=0.3 * dx / c, c_ref=c, c0=c, rho0=1000.0,
                rho0_sgx=1000.0, rho0_sgy=1000.0, pml_x_size=8, pml_y_size=8, pml_z_size=0, pml_x_alpha=2.0,
                pml_y_alpha=2.0, pml_z_alpha=0.0, p0_source_flag=1, p0_source_input=p0, sensor_mask_type=0,
                sensor_mask_index=np.arange(nx * ny) + 1, axisymmetric_flag=1)


def test_axisymmetric_matches_3d():
    nx, ny, nt, dx, c = 64, 32, 60, 1e-4, 1500.0
    a = simulate_as(_ball_inputs(nx, ny, nt, dx, c, 32), record=("p_final",), dtype=np.float64)["p_final"]
    x3 = np.arange(nx)[:, None, None] - 32
    y3 = np.arange(2 * ny)[None, :, None] - ny
    z3 = np.arange(2 * ny)[None, None, :] - ny
    inp3 = dict(Nx=nx, Ny=2 * ny, Nz=2 * ny, Nt=nt, dx=dx, dy=dx, dz=dx, dt=0.3 * dx / c, c_ref=c, c0=c,
                rho0=1000.0, rho0_sgx=1000.0, rho0_sgy=1000.0, rho0_sgz=1000.0, pml_x_size=8, pml_y_size=8,
                pml_z_size=8, pml_x_alpha=2.0, pml_y_alpha=2.0, pml_z_alpha=2.0, p0_source_flag=1,
                p0_source_input=np.exp(-(x3.astype(float) ** 2 + y3 ** 2 + z3 ** 2) / 6.0), sensor_mask_type=0,
                sensor_mask_index=np.arange(2) + 1)
    b = simulate(inp3, record=("p_final",), dtype=np.float64)["p_final"][:, ny:2 * ny, ny]
    reg = (slice(10, 54), slice(0, 20))
    err = np.linalg.norm(a[reg] - b[reg]) / np.linalg.norm(b[reg])
    assert err < 2e-2, err


def test_fp32_against_fp64_and_sources():
    """Additive pressure source near the axis in a heterogeneous nonlinear
    Stokes medium: FP32 restatement within 1e-4 of FP64."""
    rng = np.random.default_rng(4)
    nx, ny, nt, dx = 48, 24, 50, 1e-4
    c = 1500 + 30 * rng.random((nx, ny))
    inp = _ball_inputs(nx, ny, nt, dx, 1500.0, 20)
    inp.update(p0_source_flag=0, c0=c, c_ref=float(c.max()), rho0=1000 + 20 * rng.random((nx, ny)),
               nonlinear_flag=1, BonA=6.0, absorbing_flag=2, alpha_coeff=0.5)
    inp["rho0_sgx"] = inp["rho0"]
    inp["rho0_sgy"] = inp["rho0"]
    t = np.arange(30) * inp["dt"]
    sig = (5e4 * np.sin(2 * np.pi * 2e6 * t) * np.hanning(30))[None, :] * 1e-3
    inp.update(p_source_flag=30, p_source_mode=2, p_source_many=0, p_source_index=np.array([10 + nx * 0, 10 + nx * 3]) + 1,
               p_source_input=sig)
    rec = ("p", "p_max", "u", "p_final")
    a = simulate_as(inp, record=rec, dtype=np.float64)
    b = simulate_as(inp, record=rec, dtype=np.float32)
    for k in ("p", "p_max", "ux", "uy", "p_final"):
        e = np.linalg.norm(a[k] - b[k]) / np.linalg.norm(a[k])
        assert e < 1e-4, (k, e)
    assert np.abs(a["p"]).max() > 0


def test_front_end_builds_axisymmetric_datasets():
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_disc, smooth

    kg = KWaveGrid((40, 20), (1e-4, 1e-4))
    kg.set_time(10, 2e-8)
    p0 = make_disc(40, 20, 20, 1, 4)
    inp, record, _, _ = prepare(kg, {"sound_speed": 1500.0, "alpha_coeff": 0.5, "alpha_power": 1.5}, {"p0": p0},
                                {"mask": np.ones((40, 20))}, pml_size=5, axisymmetric=True)
    assert inp["axisymmetric_flag"] == 1 and inp["absorbing_flag"] == 2  # Stokes on axisymmetric grids
    m = np.zeros((40, 80))
    m[:, :20] = p0
    m[:, 21:40] = -p0[:, 1:][:, ::-1]
    m[:, 40:60] = -p0
    m[:, 61:] = p0[:, 1:][:, ::-1]
    np.testing.assert_allclose(np.asarray(inp["p0_source_input"]).reshape(40, 20), smooth(m, True)[:, :20])
    with pytest.raises(NotImplementedError):  # radial velocity sources
        prepare(kg, {"sound_speed": 1500.0}, {"u_mask": np.ones((40, 20)), "uy": np.ones((1, 5))},
                {"mask": np.ones((40, 20))}, pml_size=5, axisymmetric=True)
    ux, _, _, _ = prepare(kg, {"sound_speed": 1500.0}, {"u_mask": np.ones((40, 20)), "ux": np.ones((1, 5))},
                          {"mask": np.ones((40, 20))}, pml_size=5, axisymmetric=True)
    assert ux["ux_source_flag"] == 5 and ux["axisymmetric_flag"] == 1


def test_piston_on_axis_pressure_matches_the_closed_form():
    """kspaceFirstOrderAS_piston_analytical.m:36-140: a 1 MHz CW piston of
    5 mm radius on the axis of an axisymmetric grid (12 points per
    wavelength, CFL 0.25, PML outside the grid) gives the on-axis steady
    amplitude 2 P |sin(k (sqrt(x^2 + a^2) - x) / 2)| within 1 % (Linf over the
    axis, relative to its maximum).  PML 20 points stands in for the
    reference's 'auto' size."""
    from kwave.simulation import postprocess, prepare
    from kwave.utils import KWaveGrid
    from test_oracle_pinning import _cw

    c0, rho0, f0, a_src, mag = 1500.0, 1000.0, 1e6, 5e-3, 1e6
    ppw, cfl = 12, 0.25
    dx = c0 / (ppw * f0)
    nx, ny = int(2 * round(32e-3 / dx / 2)), int(2 * round(10e-3 / dx / 2))
    ppp = round(ppw / cfl)
    dt = 1 / (ppp * f0)
    nt = round(40e-6 / dt)
    kg = KWaveGrid((nx, ny), (dx, dx))
    kg.set_time(nt, dt)
    rgp = round(a_src / dx)
    pm = np.zeros((nx, ny))
    pm[0, :rgp] = 1
    sm = np.zeros((nx, ny))
    sm[1:, 0] = 1  # the axis
    src = {"p_mask": pm, "p": mag * _cw(np.arange(nt) * dt, f0)[None, :]}
    sensor = {"mask": sm, "record": ["p"], "record_start_index": nt - 3 * ppp + 1}
    inp, rec, start, meta = prepare(kg, {"sound_speed": c0, "density": rho0}, src, sensor,
                                    pml_size=(20, 20), pml_inside=False, axisymmetric=True)
    p = np.asarray(postprocess(simulate_as(inp, record=rec, record_start_index=start, dtype=np.float64),
                               inp, meta)["p"])
    k = int(round(f0 * p.shape[1] * dt))
    amp = 2 * np.abs(np.fft.fft(p, axis=1)[:, k]) / p.shape[1]
    x = np.arange(1, nx) * dx
    kk, a = 2 * np.pi * f0 / c0, (rgp - 0.5) * dx
    ref = mag * np.abs(2 * np.sin((kk * np.sqrt(x ** 2 + a ** 2) - kk * x) / 2))
    err = 100 * np.max(np.abs(ref - amp)) / ref.max()
    assert err <= 1.0, err
