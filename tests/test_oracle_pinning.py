"""Pin the CPU oracle to the reference's own self-consistency tests.

The reference ships no golden vectors, so the oracle is checked against the
identities its unit tests assert (k-Wave/testing/unit/):
  * kspaceFirstOrder3D_p0_vs_two_clicks.m: an initial pressure equals two
    additive-no-correction source clicks of [0.5, 0.5] / (2 c dt / dx);
  * kspaceFirstOrder3D_compare_binary_and_cuboid_sensor_mask.m;
  * kspaceFirstOrder2D_compare_labelled_and_binary_source_mask.m;
  * kspaceFirstOrder_compare_1D_2D_3D_plane_waves.m (axis symmetry);
  * kspaceFirstOrder_check_plane_wave_intensity.m (analytic time-averaged
    intensity within 1 %);
  * kspaceFirstOrder2D_check_source_scaling_p.m and _ux.m (k-space
    corrected source amplitude against a 50x finer uncorrected run, within
    1e-4);
  * kspaceFirstOrder2D_check_nonstaggered_particle_velocity.m (order of the
    regular- and staggered-grid velocity peaks);
  * kspaceFirstOrder2D_compare_binary_and_cartesian_sensor_mask.m (1e-14);
and the FP32 restatement is checked against the FP64 one (DataCast 'off').
"""
import numpy as np
import pytest

from helpers import rel_l2
from kwave.simulation import prepare
from kwave.utils import KWaveGrid, make_ball, make_disc
from oracle.kspace_oracle import simulate


def _pair(dim):
    if dim == 3:
        n = (32, 32, 32)
        p0 = make_ball(*n, 16, 16, 16, 6)
        mask = np.zeros(n)
        mask[[3, 28], :, :] = 1
    else:
        n = (64, 64)
        p0 = make_disc(*n, 32, 32, 10)
        mask = np.zeros(n)
        mask[[5, 58], :] = 1
    kg = KWaveGrid(n, (1e-4,) * dim)
    kg.make_time(1500.0, 0.234)
    kg.set_time(min(kg.Nt, 60), kg.dt)
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    sensor = {"mask": mask, "record": ["p"]}
    a, rec, _, _ = prepare(kg, medium, {"p0": p0}, sensor, smooth_p0=False, pml_alpha=0.0)
    src = {"p_mask": (p0 != 0).astype(float), "p_mode": "additive-no-correction",
           "p": np.array([[0.5, 0.5]]) / (2 * 1500.0 * kg.dt / kg.dx)}
    b, _, _, _ = prepare(kg, medium, src, sensor, smooth_p0=False, pml_alpha=0.0)
    return a, b, rec


@pytest.mark.parametrize("dim", [2, 3])
def test_p0_equals_two_clicks(dim):
    a, b, rec = _pair(dim)
    pa = simulate(a, rec, dtype=np.float64)["p"]
    pb = simulate(b, rec, dtype=np.float64)["p"]
    if dim == 3:
        # the reference's criterion: max(sensor_data(:) - sensor_data2(:)) <= 1e-14
        assert np.max(pa - pb) <= 1e-14
    # both directions, relative to the signal
    assert np.max(np.abs(pa - pb)) <= 1e-12 * np.max(np.abs(pa))


def test_cuboid_equals_binary_mask():
    n = (24, 26, 28)
    kg = KWaveGrid(n, (1e-4,) * 3)
    kg.set_time(30, 0.3e-4 / 1500)
    p0 = make_ball(*n, 12, 13, 14, 3)
    corners = np.array([[3, 4, 5, 9, 10, 8], [15, 14, 20, 20, 19, 25]]).T
    rec = ["p", "p_max", "p_rms", "u", "u_max"]
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    ic, record, _, _ = prepare(kg, medium, {"p0": p0}, {"mask": corners, "record": rec}, pml_size=4)
    ib = dict(ic)
    ib.pop("sensor_mask_corners")
    ib["sensor_mask_type"] = 0
    lin = []
    for k in range(corners.shape[1]):
        x1, y1, z1, x2, y2, z2 = corners[:, k]
        sub = np.zeros(n, dtype=bool)
        sub[x1 - 1:x2, y1 - 1:y2, z1 - 1:z2] = True
        lin.append(np.flatnonzero(sub.reshape(-1, order="F")) + 1)
    ib["sensor_mask_index"] = np.concatenate(lin)
    oc = simulate(ic, record, dtype=np.float64)
    ob = simulate(ib, record, dtype=np.float64)
    for k in ob:
        np.testing.assert_array_equal(oc[k], ob[k])


def test_labelled_equals_binary_source():
    n = (48, 40)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(60, 0.3e-4 / 1500)
    lab = np.zeros(n)
    lab[10, 5:15] = 1
    lab[30, 20:32] = 2
    lab[20:26, 35] = 3
    t = np.arange(kg.Nt) * kg.dt
    sig = np.vstack([0.5 * np.sin(2 * np.pi * 1e6 * t), 0.8 * np.sin(2 * np.pi * 2e6 * t),
                     0.2 * np.sin(2 * np.pi * 0.5e6 * t)])
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    sensor = {"mask": np.ones(n), "record": ["p_final", "p_max"]}
    il, rec, _, _ = prepare(kg, medium, {"p_mask": lab, "p": sig}, sensor, pml_size=6)
    index_mask = lab.reshape(-1, order="F")[lab.reshape(-1, order="F") != 0].astype(int)
    ib, _, _, _ = prepare(kg, medium, {"p_mask": (lab != 0).astype(float), "p": sig[index_mask - 1]}, sensor,
                          pml_size=6)
    ol = simulate(il, rec, dtype=np.float64)
    ob = simulate(ib, rec, dtype=np.float64)
    for k in ("p_final", "p_max"):
        assert np.max(np.abs(ol[k] - ob[k])) <= 1e-15 * np.max(np.abs(ob[k])) + 1e-300


@pytest.mark.parametrize("dim", [2, 3])
def test_plane_wave_axis_symmetry(dim):
    """A plane wave launched along each axis gives the same (transposed) field."""
    n = 32
    shape = (n,) * dim
    kg = KWaveGrid(shape, (1e-4,) * dim)
    kg.set_time(40, 0.3e-4 / 1500)
    t = np.arange(kg.Nt) * kg.dt
    sig = np.sin(2 * np.pi * 1.5e6 * t)[None, :] * (t[None, :] < 2e-6)
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    finals = []
    for axis in range(dim):
        mask = np.zeros(shape)
        sl = [slice(None)] * dim
        sl[axis] = 4
        mask[tuple(sl)] = 1
        inp, rec, _, _ = prepare(kg, medium, {"p_mask": mask, "p": sig},
                                 {"mask": np.ones(shape), "record": ["p_final"]}, pml_size=0)
        pf = simulate(inp, rec, dtype=np.float64)["p_final"]
        finals.append(np.moveaxis(pf, axis, 0))
    for f in finals[1:]:
        assert np.max(np.abs(f - finals[0])) <= 1e-12 * np.max(np.abs(finals[0]))


def test_fp32_restatement_tracks_fp64():
    n = (40, 36, 30)
    rng = np.random.default_rng(3)
    kg = KWaveGrid(n, (1e-4,) * 3)
    c = 1500 + 40 * rng.standard_normal(n)
    kg.set_time(40, 0.3e-4 / c.max())
    medium = {"sound_speed": c, "density": 1000 + 30 * rng.standard_normal(n), "alpha_coeff": 0.75,
              "alpha_power": 1.5, "BonA": 6.0}
    p0 = 1e5 * make_ball(*n, 20, 18, 15, 4)
    mask = np.zeros(n)
    mask[::4, ::5, ::3] = 1
    inp, rec, _, _ = prepare(kg, medium, {"p0": p0}, {"mask": mask, "record": ["p", "p_rms", "u"]}, pml_size=5)
    o64 = simulate(inp, rec, dtype=np.float64)
    o32 = simulate(inp, rec, dtype=np.float32)
    for k in o64:
        assert rel_l2(o32[k], o64[k]) < 1e-5, k


def _plane_wave_intensity_case(axis):
    """kspaceFirstOrder_check_plane_wave_intensity.m:36-200 in 2D: a 10 MHz
    plane wave of 10 W/cm^2 time-averaged intensity launched by an additive
    pressure plane (ramped over 200 samples), recorded two periods at the end
    of a 3 us run one grid point before the far PML; PML 20 (alpha 2) along
    the propagation axis, 2 (alpha 0) across it."""
    nx, nj, dx = 64, 32, 0.05e-3
    c, rho = 1500.0, 1000.0
    f0, intensity = 10e6, 10.0  # Hz, W/cm^2
    strength = np.sqrt(2 * intensity * 1e4 * rho * c)
    ppp = 30
    dt = 1.0 / f0 / (2 * ppp)
    t = np.arange(0.0, 3e-6 + dt / 2, dt)
    nt = t.size
    sig = strength * np.sin(2 * np.pi * f0 * t)
    ramp = (-np.cos(np.arange(200) * np.pi / 200) + 1) / 2
    sig[:200] *= ramp
    n = (nx, nj) if axis == 0 else (nj, nx)
    kg = KWaveGrid(n, (dx, dx))
    kg.set_time(nt, dt)
    src_mask, sens_mask = np.zeros(n), np.zeros(n)
    if axis == 0:
        src_mask[20, :] = 1
        sens_mask[nx - 20 - 2, nj // 2 - 1] = 1
        pml_size, pml_alpha = (20, 2), (2.0, 0.0)
    else:
        src_mask[:, 20] = 1
        sens_mask[nj // 2 - 1, nx - 20 - 2] = 1
        pml_size, pml_alpha = (2, 20), (0.0, 2.0)
    sensor = {"mask": sens_mask, "record": ["I", "I_avg"], "record_start_index": nt - 2 * ppp + 1}
    return prepare(kg, {"sound_speed": c, "density": rho}, {"p_mask": src_mask, "p": sig[None, :]}, sensor,
                   pml_size=pml_size, pml_alpha=pml_alpha), intensity


@pytest.mark.parametrize("axis", [0, 1])
def test_plane_wave_intensity_matches_the_source(axis):
    """The reference's analytic intensity check (error <= 1 %,
    kspaceFirstOrder_check_plane_wave_intensity.m:221-233) on the oracle:
    the time-averaged intensity at the sensor equals the launched 10 W/cm^2."""
    from kwave.simulation import postprocess

    (inp, record, start, meta), intensity = _plane_wave_intensity_case(axis)
    out = postprocess(simulate(inp, record=record, record_start_index=start, dtype=np.float64), inp, meta)
    i_avg = float(np.ravel(out["Ix_avg" if axis == 0 else "Iy_avg"])[0])
    err = 100 * abs(intensity - 1e-4 * i_avg) / intensity
    assert err <= 1.0, err


def _cw(t, f, ramp_periods=4):
    """createCWSignals.m: unit sine with a raised-cosine ramp over the first
    `ramp_periods` periods."""
    s = np.sin(2 * np.pi * f * t)
    n = int(round(ramp_periods / f / (t[1] - t[0])))
    s[:n] *= (-np.cos(np.linspace(0, np.pi, n)) + 1) * 0.5
    return s


def _source_scaling_case(fac, mode, kind="p"):
    """kspaceFirstOrder2D_check_source_scaling_p.m:36-110 (kind "p") and
    _ux.m (kind "ux": the signal divided by c rho as an x-velocity source):
    a CW line source (3 points per wavelength, CFL 0.5) on a 64 x 64 grid,
    the pressure one point before the far PML over the last three periods;
    `fac` divides the time step (50: the fine reference)."""
    pml, nx = 20, 64
    dx = 50e-3 / nx
    c = 1500.0
    freq = c / (3 * dx)
    ppp = round(3 / 0.5)
    dt = 1 / (ppp * freq)
    nt = round(50e-6 / dt)
    dt, nt, ppp = dt / fac, nt * fac, ppp * fac
    kg = KWaveGrid((nx, nx), (dx, dx))
    kg.set_time(nt, dt)
    pm = np.zeros((nx, nx))
    pm[pml, pml:nx - pml] = 1
    sm = np.zeros((nx, nx))
    sm[nx - pml - 1, nx // 2 - 1] = 1
    sig = _cw(np.arange(nt) * dt, freq)[None, :]
    if kind == "p":
        src = {"p_mask": pm, "p": sig, "p_mode": mode}
    else:
        src = {"u_mask": pm, "ux": sig / (c * 1000.0), "u_mode": mode}
    sensor = {"mask": sm, "record": ["p"], "record_start_index": nt - 3 * ppp + 1}
    return prepare(kg, {"sound_speed": c, "density": 1000.0}, src, sensor, pml_size=pml), freq, dt


def _cw_amplitude(x, freq, dt):
    """extractAmpPhase.m with a rectangular window and no padding: the
    single-sided spectrum at the bin of `freq` (three whole periods)."""
    x = np.ravel(x)
    k = int(round(freq * x.size * dt))
    return 2 * abs(np.fft.fft(x)[k]) / x.size


def source_scaling_reference_amplitude(kind="p"):
    (inp, record, start, _), freq, dt = _source_scaling_case(50, "additive-no-correction", kind)
    out = simulate(inp, record=record, record_start_index=start, dtype=np.float64)
    return _cw_amplitude(out["p"], freq, dt)


@pytest.mark.parametrize("kind", ["p", "ux"])
def test_kspace_corrected_source_scaling(kind):
    """The reference's source-scaling checks (error <= 1e-4,
    kspaceFirstOrder2D_check_source_scaling_p.m:112-118, _ux.m): the k-space
    corrected additive source at the coarse step gives the amplitude of an
    uncorrected source at a 50x finer step."""
    fine = source_scaling_reference_amplitude(kind)
    (inp, record, start, _), freq, dt = _source_scaling_case(1, "additive", kind)
    out = simulate(inp, record=record, record_start_index=start, dtype=np.float64)
    err = abs(_cw_amplitude(out["p"], freq, dt) - fine) / fine
    assert err <= 1e-4, err


def test_non_staggered_velocity_lies_between_staggered_points():
    """kspaceFirstOrder2D_check_nonstaggered_particle_velocity.m:36-101: for
    an outgoing wave in an absorbing medium, recorded at two adjacent points
    along x, the peaks of u_x on the regular grid (at the point) and on the
    staggered grid (half a cell further out) fall in that order: each
    smaller and no earlier than the one before."""
    from kwave.simulation import postprocess

    n = (128, 128)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    medium = {"sound_speed": 1500.0, "density": 1000.0, "alpha_coeff": 0.75, "alpha_power": 1.5}
    kg.make_time(1500.0, cfl=0.1, t_end=6e-6)
    mask = np.zeros(n)
    mask[64 + 40 - 1, 64 - 1] = 1
    mask[64 + 40, 64 - 1] = 1
    p0 = 5 * make_disc(n[0], n[1], 64, 64, 5)
    inp, record, start, meta = prepare(kg, medium, {"p0": p0}, {"mask": mask, "record": ["p", "u", "u_non_staggered"]})
    out = postprocess(simulate(inp, record=record, record_start_index=start, dtype=np.float64), inp, meta)
    uns, us = np.asarray(out["ux_non_staggered"]), np.asarray(out["ux"])
    seq = [uns[0], us[0], uns[1], us[1]]
    peaks = [float(s.max()) for s in seq]
    when = [int(np.argmax(s)) for s in seq]
    assert peaks[0] > peaks[1] > peaks[2] > peaks[3], peaks
    assert when[0] <= when[1] <= when[2] <= when[3], when


def test_binary_and_cartesian_sensors_agree():
    """kspaceFirstOrder2D_compare_binary_and_cartesian_sensor_mask.m:36-150:
    Cartesian sensor points placed on grid nodes give, with linear
    interpolation and with the nearest-point mapping, the outputs of the
    same points as a binary mask reordered to the points' order (relative
    max error 1e-14), for p, u, u on the regular grid, their max / min / rms
    and the intensity.  A one-point-wide ring (a disc less a smaller disc)
    stands in for makeCircle."""
    from kwave.simulation import postprocess

    n = (128, 128)
    dx = 25e-3 / n[0]
    kg = KWaveGrid(n, (dx, dx))
    c = 1500 * np.ones(n)
    c[n[0] // 2 - 1:, :] = 2000
    rho = 1000 * np.ones(n)
    rho[n[0] // 2 - 1:, :] = 1200
    kg.make_time(c)
    p0 = np.zeros(n)
    p0[21, n[1] // 4 - 1:3 * n[1] // 4] = 1
    ring = make_disc(n[0], n[1], n[0] // 2, n[1] // 2, n[0] // 2 - 10) - make_disc(
        n[0], n[1], n[0] // 2, n[1] // 2, n[0] // 2 - 11)
    jj, ii = np.nonzero(ring.T)  # MATLAB find order: x fastest
    cart = np.stack([kg.vec(0)[ii], kg.vec(1)[jj]])
    record = ["p", "p_max", "p_min", "p_rms", "u", "u_max", "u_min", "u_rms", "u_non_staggered", "I", "I_avg"]
    medium = {"sound_speed": c, "density": rho}
    runs = {}
    for name, mask, interp in (("linear", cart, "linear"), ("nearest", cart, "nearest"), ("binary", cart, None)):
        kw = {"cart_interp": interp} if interp else {}
        if interp is None:
            from kwave.utils import cart2grid

            mask = cart2grid(kg, cart)[0]
        inp, rec, start, meta = prepare(kg, medium, {"p0": p0}, {"mask": mask, "record": list(record)}, **kw)
        runs[name] = postprocess(simulate(inp, record=rec, record_start_index=start, dtype=np.float64), inp, meta)
        if interp is None:  # binary outputs come in grid order: reorder to the points' order
            from kwave.utils import reorder_binary_sensor_data

            order = cart2grid(kg, cart)[1]
            runs[name] = {k: (reorder_binary_sensor_data(np.asarray(v), order) if np.ndim(v) and
                              np.shape(v)[0] == cart.shape[1] else v) for k, v in runs[name].items()}
    keys = [k for k in runs["binary"] if k in runs["linear"] and k in runs["nearest"]]
    assert {"p", "p_max", "ux", "uy_rms", "ux_non_staggered", "Ix_avg"} <= set(keys), keys
    for k in keys:
        b = np.asarray(runs["binary"][k], dtype=np.float64)
        for other in ("linear", "nearest"):
            o = np.asarray(runs[other][k], dtype=np.float64)
            err = np.max(np.abs(o - b)) / np.max(np.abs(b))
            assert err <= 1e-14, (k, other, err)
