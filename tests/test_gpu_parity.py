"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on
the same seeded inputs.

Tolerances (relative L2 over each output array): 1e-5 for linear lossless
runs and 1e-4 otherwise, against the FP64 oracle (the reference with
DataCast 'off'); the FP32 oracle is checked at the same bars.
"""
import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het, compare, oracle_outputs, rel_l2

pytestmark = pytest.mark.gpu

TOL_LOSSLESS = 1e-5
TOL = 1e-4


def _solve(inp, record, start=1):
    from kwave import _lib

    return _lib.solve(inp, record=record, start_index=start)


def _check(inp, record, tol, start=1):
    gpu = _solve(inp, record, start)
    for dt in (np.float64, np.float32):
        ora = oracle_outputs(inp, record, start, dtype=dt)
        errs = compare(gpu, ora)
        assert errs, "no common outputs"
        bad = {k: v for k, v in errs.items() if not v <= tol}
        assert not bad, f"{np.dtype(dt).name} oracle: {bad}"
    return gpu


def test_2d_p0_lossless_all_records():
    inp, record, start, _ = case_2d_p0()
    _check(inp, record, TOL_LOSSLESS)


def test_2d_p0_odd_sizes():
    inp, record, start, _ = case_2d_p0(n=(45, 50), nt=60, record=("p", "p_max", "u", "p_final"))
    _check(inp, record, TOL_LOSSLESS)


def test_3d_p0_lossless():
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_ball

    n = (32, 30, 27)
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(50, 0.3e-4 / 1500)
    p0 = make_ball(*n, 16, 15, 14, 4)
    mask = np.zeros(n)
    mask[4:28:5, 3:27:4, 2:25:6] = 1
    inp, record, start, _ = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": p0},
                                    {"mask": mask, "record": ["p", "u", "p_max", "p_rms", "p_final",
                                                              "u_final", "p_min_all"]}, pml_size=5)
    _check(inp, record, TOL_LOSSLESS)


def test_3d_heterogeneous_absorbing_nonlinear_additive_source():
    inp, record, start, _ = case_3d_het()
    _check(inp, record, TOL)


def test_3d_stokes_dirichlet_source():
    inp, record, start, _ = case_3d_het(stokes=True, p_mode="dirichlet", nonlinear=False)
    _check(inp, record, TOL)


def test_3d_additive_no_correction_many_signals():
    inp, record, start, _ = case_3d_het(p_mode="additive-no-correction", many=True, absorbing=False)
    _check(inp, record, TOL)


def test_3d_additive_many_signals():
    inp, record, start, _ = case_3d_het(p_mode="additive", many=True, nonlinear=False)
    _check(inp, record, TOL)


def test_record_start_index():
    inp, record, start, _ = case_2d_p0(record=("p", "p_max", "p_rms", "u_rms"))
    _check(inp, record, TOL_LOSSLESS, start=17)


@pytest.mark.parametrize("mode", ["dirichlet", "additive", "additive-no-correction"])
def test_2d_velocity_sources(mode):
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, tone_burst

    n = (48, 40)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(70, 0.3e-4 / 1500)
    umask = np.zeros(n)
    umask[10, 12:28] = 1
    sig = tone_burst(1 / kg.dt, 3e6, 2)
    source = {"u_mask": umask, "ux": sig, "uy": 0.5 * sig, "u_mode": mode}
    smask = np.zeros(n)
    smask[20:40:3, 5:35:4] = 1
    inp, record, start, _ = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, source,
                                    {"mask": smask, "record": ["p", "u", "u_max"]}, pml_size=6)
    _check(inp, record, TOL_LOSSLESS)


def test_cuboid_equals_binary_mask():
    """kspaceFirstOrder3D_compare_binary_and_cuboid_sensor_mask.m: the same
    points recorded through cuboid corners and through a binary mask."""
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_ball

    n = (30, 32, 36)
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(40, 0.3e-4 / 1500)
    p0 = make_ball(*n, 15, 16, 18, 3)
    corners = np.array([[4, 5, 6, 10, 12, 9], [20, 18, 25, 24, 22, 30]]).T
    rec = ["p", "p_max", "u"]
    inp_c, record, _, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": p0},
                                     {"mask": corners, "record": rec}, pml_size=5)
    mask = np.zeros(n)
    lin = []
    for k in range(corners.shape[1]):
        x1, y1, z1, x2, y2, z2 = corners[:, k]
        sub = np.zeros(n, dtype=bool)
        sub[x1 - 1:x2, y1 - 1:y2, z1 - 1:z2] = True
        lin.append(np.flatnonzero(sub.reshape(-1, order="F")) + 1)
    inp_b = dict(inp_c)
    inp_b.pop("sensor_mask_corners")
    inp_b["sensor_mask_type"] = 0
    inp_b["sensor_mask_index"] = np.concatenate(lin)
    a = _solve(inp_c, record)
    b = _solve(inp_b, record)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_output_sizes_and_errors():
    from kwave import _lib

    inp, record, start, _ = case_2d_p0()
    bad = dict(inp)
    bad["sensor_mask_index"] = np.array([0, 5])
    with pytest.raises(_lib.KwaveError):
        _solve(bad, record)
    bad = dict(inp)
    bad["Nx"] = 11 * 8  # a prime factor above 7
    with pytest.raises(_lib.KwaveError, match="factor"):
        _solve(bad, record)


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 64, 64), (64, 128, 128)])
def test_3d_compile_time_sizes_het_absorbing(shape):
    """Grid edges served by the compile-time FFT engine."""
    inp, record, start, _ = case_3d_het(n=shape, nt=30, record=("p", "p_max", "p_rms", "u", "p_final"))
    _check(inp, record, TOL)


def test_2d_compile_time_sizes():
    inp, record, start, _ = case_2d_p0(n=(128, 256), nt=60, record=("p", "p_max", "u", "p_final", "u_final"))
    _check(inp, record, TOL_LOSSLESS)


def test_2d_nonlinear_absorbing_512():
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_disc

    n = (512, 64)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(40, 0.3e-4 / 1600)
    rng = np.random.default_rng(11)
    c = 1500 + 30 * rng.standard_normal(n)
    medium = {"sound_speed": c, "density": 1000.0, "alpha_coeff": 0.5, "alpha_power": 1.3, "BonA": 5.0}
    p0 = 1e5 * make_disc(n[0], n[1], 256, 32, 6)
    mask = np.zeros(n)
    mask[::17, ::9] = 1
    inp, record, start, _ = prepare(kg, medium, {"p0": p0}, {"mask": mask, "record": ["p", "p_rms", "u_max"]},
                                    pml_size=10)
    _check(inp, record, TOL)


@pytest.mark.parametrize("n", [(75, 81), (100, 108), (243, 250), (729, 90), (1000, 64), (972, 125)])
def test_2d_compile_time_mixed_radix_sizes(n):
    """Compile-time FFT kernels of 2^a 3^b 5^c lengths (radix-3 and -5 stages,
    line counts that are not multiples of 4, up to 1024 points)."""
    inp, record, start, _ = case_2d_p0(n=n, nt=30, record=("p", "p_max", "u", "p_final"))
    _check(inp, record, TOL_LOSSLESS)


@pytest.mark.parametrize("n", [(72, 75, 80), (81, 90, 64)])
def test_3d_compile_time_mixed_radix_sizes(n):
    inp, record, start, _ = case_3d_het(n=n, nt=24, record=("p", "p_rms", "u"))
    _check(inp, record, TOL)


@pytest.mark.parametrize("nz", [80, 81, 96, 125, 144, 162, 192, 243, 250])
def test_tma_last_axis_operator_on_multi_stage_lengths(nz):
    """The TMA-fed last-axis operator on 2^a 3^b 5^c lengths other than 64,
    128 and 256 (forward transform, operator and inverse through shared
    memory, no register hand-off), against the oracle."""
    inp, record, start, _ = case_3d_het(n=(32, 30, nz), nt=12, record=("p", "p_max", "p_rms", "u", "p_final"))
    _check(inp, record, TOL)


@pytest.mark.parametrize("n", [(56, 42), (112, 49), (98, 70)])
def test_2d_radix7_sizes(n):
    """Edges with a factor 7 (the runtime FFT engine's radix-7 stage)."""
    inp, record, start, _ = case_2d_p0(n=n, nt=30, record=("p", "p_max", "u", "p_final"))
    _check(inp, record, TOL_LOSSLESS)


def test_3d_radix7_sizes():
    inp, record, start, _ = case_3d_het(n=(28, 36, 35), nt=24, record=("p", "p_rms", "u", "p_final"))
    _check(inp, record, TOL)


def test_2d_u_non_staggered():
    """u shifted to the regular grid (kspaceFirstOrder_extractSensorData.m:109-120)."""
    inp, record, start, _ = case_2d_p0(n=(64, 48), nt=50, record=("p", "u", "u_non_staggered"))
    gpu = _check(inp, record, TOL_LOSSLESS)
    assert "ux_non_staggered" in gpu and "uy_non_staggered" in gpu
    assert not np.allclose(gpu["ux_non_staggered"], gpu["ux"])  # the shift moved the samples


@pytest.mark.parametrize("n", [(32, 30, 36), (72, 60, 64), (64, 64, 64)])
def test_3d_u_non_staggered(n):
    inp, record, start, _ = case_3d_het(n=n, nt=30, record=("p", "u_non_staggered", "u_rms"))
    gpu = _check(inp, record, TOL, start=4)
    assert {"ux_non_staggered", "uy_non_staggered", "uz_non_staggered"} <= set(gpu)


def test_intensity_from_the_gpu_path():
    """sensor.record {'I', 'I_avg'}: p and u_non_staggered from the GPU,
    intensity on the host (kspaceFirstOrder_saveIntensity.m:42-75), against the
    same post-processing of the oracle's outputs."""
    from kwave import _lib
    from kwave.simulation import postprocess, prepare
    from kwave.utils import KWaveGrid, make_disc

    n = (64, 64)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(80, 0.3e-4 / 1500)
    mask = np.zeros(n)
    mask[40, 20:44] = 1
    sensor = {"mask": mask, "record": ["p", "I", "I_avg"]}
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0},
                                       {"p0": 2 * make_disc(*n, 32, 32, 5)}, sensor, pml_size=8)
    assert "u_non_staggered" in record
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(oracle_outputs(inp, record, start, dtype=np.float64), inp, meta)
    for k in ("Ix", "Iy", "Ix_avg", "Iy_avg"):
        assert rel_l2(gpu[k], ora[k]) < TOL, k


def test_3d_cartesian_linear_interpolation():
    """Cartesian sphere sensor with 'CartInterp' linear: the vertex series
    from the GPU, interpolated and reduced on the host, against the oracle's
    through the same postprocess()."""
    from kwave import _lib
    from kwave.simulation import postprocess, prepare
    from kwave.utils import KWaveGrid, make_ball, make_cart_sphere

    n = (40, 36, 32)
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(70, 0.3e-4 / 1500)
    pts = make_cart_sphere(1.1e-3, 40)
    sensor = {"mask": pts, "record": ["p", "p_max", "p_rms", "u", "u_min", "I_avg"]}
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0},
                                       {"p0": 2 * make_ball(*n, 20, 18, 16, 4)}, sensor, pml_size=6,
                                       cart_interp="linear")
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(oracle_outputs(inp, record, start, dtype=np.float64), inp, meta)
    tol = {k: TOL_LOSSLESS for k in ("p", "p_max", "p_rms", "ux", "uy", "uz", "ux_min", "uz_min")}
    tol.update(Ix_avg=TOL, Iz_avg=TOL)  # products of two series, shifted on the host
    assert set(tol) <= set(gpu) and gpu["p"].shape == (40, 70)
    bad = {k: rel_l2(gpu[k], ora[k]) for k in tol if not rel_l2(gpu[k], ora[k]) <= tol[k]}
    assert not bad, bad


def test_2d_cartesian_circle_linear_interpolation():
    """The 2D Cartesian-circle configuration (50 points, 'CartInterp' linear,
    the in-memory default): per-point series and reductions formed on the
    device each step; full-grid outputs alongside."""
    from kwave import _lib
    from kwave.simulation import postprocess, prepare
    from kwave.utils import KWaveGrid, make_cart_circle, make_disc

    n = (128, 128)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(150, 0.3e-4 / 1500)
    p0 = 5 * make_disc(*n, 64, 60, 5) + 3 * make_disc(*n, 50, 80, 4)
    sensor = {"mask": make_cart_circle(4.5e-3, 50), "record": ["p", "p_max", "p_min", "p_rms", "u_rms", "u",
                                                                 "p_final", "p_max_all"]}
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": p0}, sensor,
                                       pml_size=20, cart_interp="linear")
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(oracle_outputs(inp, record, start, dtype=np.float64), inp, meta)
    assert gpu["p"].shape == (50, 150) and gpu["p_max_all"].shape == n
    bad = {k: rel_l2(gpu[k], ora[k]) for k in ora if not rel_l2(gpu[k], ora[k]) <= TOL_LOSSLESS}
    assert not bad, bad


@pytest.mark.parametrize("interp", ["linear", "nearest"])
def test_config_2d_two_discs_cartesian_circle(interp):
    """The reference's CPU-runnable case: 128 x 128, dx 0.1 mm, lossless
    homogeneous, PML 20, two smoothed discs of p0, a 50-point Cartesian circle
    of radius 4 mm (linear: the in-memory default; nearest: the file path),
    CFL 0.3 to 8 us."""
    from kwave import _lib
    from kwave.simulation import postprocess, prepare
    from kwave.workloads import two_disc_2d

    kg, medium, source, sensor = two_disc_2d()
    sensor["record"] = ["p", "p_max", "p_rms"]
    inp, record, start, meta = prepare(kg, medium, source, sensor, cart_interp=interp)
    assert inp["Nt"] == kg.Nt and kg.Nt > 300
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(oracle_outputs(inp, record, start, dtype=np.float64), inp, meta)
    assert gpu["p"].shape == (50, kg.Nt)
    bad = {k: rel_l2(gpu[k], ora[k]) for k in ora if not rel_l2(gpu[k], ora[k]) <= TOL_LOSSLESS}
    assert not bad, bad


def test_slabs_on_two_streams_give_identical_results():
    """The y-inverse / row kernel / y-forward chains split into z slabs on two
    streams (the default for large 3D grids) give bit-identical outputs."""
    import os

    from kwave import _lib

    inp, record, start, _ = case_3d_het(n=(64, 48, 40), nt=30, record=("p", "p_max", "p_rms", "u", "p_final"))
    whole = _lib.solve(inp, record, start_index=start)
    old = {k: os.environ.get(k) for k in ("KWAVE_B200_SLAB", "KWAVE_B200_SLAB_STREAMS")}
    os.environ.update(KWAVE_B200_SLAB="11", KWAVE_B200_SLAB_STREAMS="2")
    try:
        split = _lib.solve(inp, record, start_index=start)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    for k in whole:
        np.testing.assert_array_equal(split[k], whole[k], err_msg=k)


TMA_Y_LENGTHS = [72, 75, 80, 81, 90, 96, 100, 108, 120, 125, 135, 144, 150, 160, 162, 180, 192, 200, 216, 225,
                 240, 243, 250]


@pytest.mark.parametrize("ny", TMA_Y_LENGTHS)
def test_tma_y_pass_matches_plain_y_pass(ny):
    """The TMA-fed y pass on 2^a 3^b 5^c lengths other than powers of two
    (tiles of an even number of lines, so every tile starts 16-byte aligned)
    gives bit for bit the outputs of the plain column kernels."""
    import os

    from kwave import _lib

    inp, record, start, _ = case_3d_het(n=(64, ny, 24), nt=6, record=("p", "p_max", "p_rms", "u", "p_final"))
    tma = _lib.solve(inp, record, start_index=start)
    old = os.environ.get("KWAVE_B200_NO_TMA")
    os.environ["KWAVE_B200_NO_TMA"] = "1"
    try:
        plain = _lib.solve(inp, record, start_index=start)
    finally:
        if old is None:
            os.environ.pop("KWAVE_B200_NO_TMA", None)
        else:
            os.environ["KWAVE_B200_NO_TMA"] = old
    for k in plain:
        np.testing.assert_array_equal(tma[k], plain[k], err_msg=k)


def test_tma_y_pass_192_against_oracle():
    inp, record, start, _ = case_3d_het(n=(64, 192, 24), nt=16, record=("p", "p_max", "u", "p_final"))
    _check(inp, record, TOL)


@pytest.mark.parametrize("axis", [0, 1])
def test_plane_wave_intensity_on_the_gpu(axis):
    """The reference's analytic plane-wave intensity check (10 W/cm^2 within
    1 %, kspaceFirstOrder_check_plane_wave_intensity.m:221-233) through the
    GPU path, and its I_avg against the oracle's."""
    from kwave import _lib
    from kwave.simulation import postprocess
    from test_oracle_pinning import _plane_wave_intensity_case

    (inp, record, start, meta), intensity = _plane_wave_intensity_case(axis)
    key = "Ix_avg" if axis == 0 else "Iy_avg"
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(oracle_outputs(inp, record, start, dtype=np.float64), inp, meta)
    i_gpu = float(np.ravel(gpu[key])[0])
    assert 100 * abs(intensity - 1e-4 * i_gpu) / intensity <= 1.0
    assert abs(i_gpu - float(np.ravel(ora[key])[0])) <= TOL * abs(i_gpu)


def test_kspace_corrected_source_scaling_on_the_gpu():
    """The reference's source-scaling check (kspaceFirstOrder2D_check_source_scaling_p.m,
    error <= 1e-4) with the coarse, k-space corrected run on the GPU and the
    fine uncorrected reference from the oracle."""
    from kwave import _lib
    from test_oracle_pinning import _cw_amplitude, _source_scaling_case, source_scaling_reference_amplitude

    fine = source_scaling_reference_amplitude()
    (inp, record, start, _), freq, dt = _source_scaling_case(1, "additive")
    gpu = _lib.solve(inp, record=record, start_index=start)
    err = abs(_cw_amplitude(gpu["p"], freq, dt) - fine) / fine
    assert err <= 1e-4, err
