"""Axisymmetric solver on the GPU (kspaceFirstOrderAS.m) against the
axisymmetric oracle, on the TMA and non-TMA radial sizes, through kw_solve,
the input file and the front end."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL_LOSSLESS = 1e-5
TOL = 1e-4


def _inputs(nx, ny, nt, het=False, seed=3):
    rng = np.random.default_rng(seed)
    dx = 1e-4
    c = 1500 + 40 * rng.random((nx, ny)) if het else 1500.0
    rho = 1000 + 30 * rng.random((nx, ny)) if het else 1000.0
    c_ref = float(np.max(c))
    xx = np.arange(nx)[:, None] - nx // 2
    yy = np.arange(ny)[None, :]
    p0 = 2 * np.exp(-(xx.astype(float) ** 2 + (yy - 3.0) ** 2) / 5.0)
    mask = np.zeros((nx, ny))
    mask[::3, ::2] = 1
    return dict(Nx=nx, Ny=ny, Nz=1, Nt=nt, dx=dx, dy=dx, dz=0.0, dt=0.3 * dx / c_ref, c_ref=c_ref, c0=c,
                rho0=rho, rho0_sgx=rho, rho0_sgy=rho, pml_x_size=6, pml_y_size=6, pml_z_size=0,
                pml_x_alpha=2.0, pml_y_alpha=2.0, pml_z_alpha=0.0, p0_source_flag=1, p0_source_input=p0,
                sensor_mask_type=0, sensor_mask_index=np.flatnonzero(mask.reshape(-1, order="F")) + 1,
                axisymmetric_flag=1)


def _check(inp, record, tol, start=1):
    from kwave import _lib
    from oracle.kspace_oracle_as import simulate_as

    gpu = _lib.solve(inp, record=record, start_index=start)
    ora = simulate_as(inp, record=record, record_start_index=start, dtype=np.float64)
    errs = {k: rel_l2(gpu[k], ora[k]) for k in ora if k in gpu}
    assert errs and max(errs.values()) <= tol, errs
    for k in ("p_final", "ux_final", "p_max_all"):
        if k in gpu:
            assert gpu[k].shape == (inp["Nx"], inp["Ny"]), k
    return gpu


@pytest.mark.parametrize("ny", [64, 20])  # expanded radial lengths 256 (TMA) and 80
def test_p0_lossless(ny):
    inp = _inputs(48, ny, 60)
    _check(inp, ("p", "p_max", "p_rms", "u", "u_max", "p_final", "u_final", "p_max_all", "p_min_all"),
           TOL_LOSSLESS)


def test_het_nonlinear_stokes_sources():
    base = _inputs(64, 32, 70, het=True)
    base.update(p0_source_flag=0, nonlinear_flag=1, BonA=5.0, absorbing_flag=2, alpha_coeff=0.75)
    t = np.arange(40) * base["dt"]
    sig = 1e3 * np.sin(2 * np.pi * 2e6 * t) * np.hanning(40)
    idx = np.array([20 + 64 * 0, 20 + 64 * 4, 33 + 64 * 9]) + 1  # on the axis and off it
    rec = ("p", "p_max", "p_min", "u", "p_final")
    for mode, many in ((2, 0), (1, 1), (0, 0), (2, 1)):
        inp = dict(base)
        s = sig[None, :] * (1 + 0.2 * np.arange(3)[:, None]) if many else sig[None, :]
        # scaled density increments (kspaceFirstOrder_scaleSourceTerms.m): about 1e-3 kg/m^3
        inp.update(p_source_flag=40, p_source_mode=mode, p_source_many=many, p_source_index=idx,
                   p_source_input=1e-6 * s)
        _check(inp, rec, TOL, start=5)


def test_input_file_matches_solve(tmp_path):
    from kwave import _lib, h5io

    inp = _inputs(48, 32, 40, het=True)
    rec = ("p", "p_final", "u_max")
    fin, fout = tmp_path / "as_in.h5", tmp_path / "as_out.h5"
    h5io.write_input_file(fin, inp)
    _lib.run_file(fin, fout, rec)
    got = h5io.read_output_file(fout, 2)
    want = _lib.solve(inp, record=rec)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


@pytest.mark.parametrize("inside", [True, False])
def test_front_end(inside):
    from kwave import kspaceFirstOrderAS
    from kwave.simulation import postprocess, prepare
    from kwave.utils import KWaveGrid, make_disc
    from oracle.kspace_oracle_as import simulate_as

    kg = KWaveGrid((64, 32), (1e-4, 1e-4))
    kg.set_time(50, 0.3e-4 / 1500)
    p0 = 3 * make_disc(64, 32, 32, 1, 5)
    sensor = {"mask": np.pad(np.ones((1, 10)), ((40, 23), (0, 22))), "record": ["p", "p_max"]}
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    sensor["record"] = ["p", "p_max", "p_final"]
    out = kspaceFirstOrderAS(kg, medium, {"p0": p0}, sensor, pml_size=8, pml_inside=inside)
    inp, record, start, meta = prepare(kg, medium, {"p0": p0}, sensor, pml_size=8, axisymmetric=True,
                                       pml_inside=inside)
    ora = postprocess(simulate_as(inp, record=record, dtype=np.float64), inp, meta)
    assert out["p_final"].shape == (64, 32)
    for k in ("p", "p_max", "p_final"):
        assert rel_l2(out[k], ora[k]) <= TOL_LOSSLESS, k


def test_rejects_what_it_does_not_run():
    from kwave import _lib

    inp = _inputs(32, 16, 10)
    bad = dict(inp, absorbing_flag=1, alpha_coeff=0.5, alpha_power=1.5)
    with pytest.raises(_lib.KwaveError, match="Stokes"):
        _lib.solve(bad, record=("p",))
    with pytest.raises(_lib.KwaveError, match="u_non_staggered"):
        _lib.solve(inp, record=("u_non_staggered",))


def test_tester_axisymmetric_case():
    """The reference harness's axisymmetric configuration (kWaveTester.m
    test_dim 4, grid type 1): 128 x 64, PML 20 / 10 inside, heterogeneity x1.3
    in the far half of a disc of radius 10, Stokes absorption with y = 2,
    B/A 6, an initial-pressure disc of radius 5, CFL 0.1."""
    from kwave import _lib
    from kwave.simulation import postprocess, prepare
    from kwave.utils import KWaveGrid, make_disc
    from oracle.kspace_oracle_as import simulate_as

    nx, ny = 128, 64
    dx = 40e-3 / nx
    kg = KWaveGrid((nx, ny), (dx, dx))
    het = make_disc(nx, 2 * ny, nx // 2, ny // 2, 10)[:, ny:] == 1
    medium = {"sound_speed": np.where(het, 1540 * 1.3, 1540.0), "density": np.where(het, 1300.0, 1000.0),
              "BonA": np.where(het, 7.8, 6.0), "alpha_coeff": np.where(het, 0.975, 0.75), "alpha_power": 2.0,
              "alpha_mode": "stokes"}
    kg.make_time(medium["sound_speed"], cfl=0.1)
    kg.set_time(120, kg.dt)
    mask = np.zeros((nx, ny))
    mask[::4, ::3] = 1
    sensor = {"mask": mask, "record": ["p", "p_max", "u", "p_final"]}
    src = {"p0": 1e6 * make_disc(nx, ny, nx // 2, ny // 2, 5)}
    inp, record, start, meta = prepare(kg, medium, src, sensor, pml_size=(20, 10), axisymmetric=True)
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(simulate_as(inp, record=record, record_start_index=start, dtype=np.float64), inp, meta)
    errs = {k: rel_l2(gpu[k], ora[k]) for k in ora}
    assert max(errs.values()) <= TOL, errs


@pytest.mark.parametrize("mode", [2, 1, 0])
def test_axial_velocity_sources(mode):
    """A piston: axial velocity on a disc of the axial plane, the usual
    axisymmetric transducer model (kspaceFirstOrderAS.m:785-830)."""
    base = _inputs(64, 32, 60, het=True)
    base.update(p0_source_flag=0)
    t = np.arange(35) * base["dt"]
    sig = 1e-3 * np.sin(2 * np.pi * 2e6 * t) * np.hanning(35)
    idx = np.array([10 + 64 * y for y in range(6)]) + 1  # x = 10, radius 0..5 (the axis included)
    many = 1 if mode == 1 else 0
    s = sig[None, :] * (1 + 0.1 * np.arange(6)[:, None]) if many else sig[None, :]
    base.update(ux_source_flag=35, u_source_mode=mode, u_source_many=many, u_source_index=idx, ux_source_input=s)
    gpu = _check(base, ("p", "u", "p_max", "p_final"), TOL)
    assert np.abs(gpu["p"]).max() > 0


def test_piston_on_axis_pressure_on_the_gpu():
    """The reference's analytic piston check (kspaceFirstOrderAS_piston_analytical.m,
    Linf <= 1 %) through the GPU path: PML 22 axial / 20 radial outside the
    grid, so the expanded grid is 300 x 4 * 100 points."""
    from kwave import _lib
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
    sm[1:, 0] = 1
    src = {"p_mask": pm, "p": mag * _cw(np.arange(nt) * dt, f0)[None, :]}
    sensor = {"mask": sm, "record": ["p"], "record_start_index": nt - 3 * ppp + 1}
    inp, rec, start, meta = prepare(kg, {"sound_speed": c0, "density": rho0}, src, sensor,
                                    pml_size=(22, 20), pml_inside=False, axisymmetric=True)
    assert (int(inp["Nx"]), int(inp["Ny"])) == (300, 100)
    p = np.asarray(postprocess(_lib.solve(inp, record=rec, start_index=start), inp, meta)["p"])
    k = int(round(f0 * p.shape[1] * dt))
    amp = 2 * np.abs(np.fft.fft(p, axis=1)[:, k]) / p.shape[1]
    x = np.arange(1, nx) * dx
    kk, a = 2 * np.pi * f0 / c0, (rgp - 0.5) * dx
    ref = mag * np.abs(2 * np.sin((kk * np.sqrt(x ** 2 + a ** 2) - kk * x) / 2))
    assert 100 * np.max(np.abs(ref - amp)) / ref.max() <= 1.0
