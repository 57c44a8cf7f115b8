"""Host-side restatements of the reference's MATLAB pre-processing."""
import numpy as np
import pytest

from kwave.simulation import fourier_shift, prepare, staggered_density
from kwave.utils import (KWaveGrid, cart2grid, make_ball, make_cart_circle, make_cart_sphere, make_dim, make_disc,
                         matlab_round, reorder_binary_sensor_data, smooth, tone_burst)


def test_matlab_round_halves_away_from_zero():
    np.testing.assert_array_equal(matlab_round([0.5, 1.5, 2.5, -0.5, -1.5]), [1, 2, 3, -1, -2])


def test_make_dim_has_exact_zero_and_nyquist_sign():
    k = make_dim(8, 1.0)
    assert k[4] == 0.0 and k[0] == -np.pi  # kWaveGrid.m:786-792
    k = make_dim(9, 1.0)
    assert k[4] == 0.0 and np.isclose(k[-1], 2 * np.pi * 4 / 9)


def test_make_disc_and_ball_centres():
    d = make_disc(20, 30, 5, 7, 3)
    assert d[4, 6] == 1 and d.sum() == 29  # 1-based centre (5, 7), radius 3 -> 29 points
    b = make_ball(16, 16, 16, 8, 9, 10, 2)
    assert b[7, 8, 9] == 1 and b.sum() == 33


def test_cart2grid_and_reorder_roundtrip():
    kg = KWaveGrid((64, 64), (1e-4, 1e-4))
    pts = make_cart_circle(2e-3, 12)
    mask, order, reorder = cart2grid(kg, pts)
    assert mask.sum() == 12
    idx = np.flatnonzero(mask.reshape(-1, order="F"))
    data = np.arange(12)[:, None] * np.ones((1, 3))
    # data recorded in mask order comes back in Cartesian order
    recorded = np.empty_like(data)
    point_of_slot = reorder - 1
    recorded[:] = data[point_of_slot]
    back = reorder_binary_sensor_data(recorded, reorder)
    np.testing.assert_array_equal(back, data)
    s = make_cart_sphere(1.0, 50)
    assert np.allclose(np.linalg.norm(s, axis=0), 1.0)


def test_tone_burst_shape():
    fs, f0 = 50e6, 1e6
    sig = tone_burst(fs, f0, 3)
    n = int(np.floor(3 / f0 * fs + 1e-9)) + 1
    assert sig.shape == (1, n)
    assert abs(sig[0, 0]) < 1e-12 and np.max(np.abs(sig)) < 1.0


def test_smooth_keeps_mean_and_restores_max():
    rng = np.random.default_rng(0)
    a = rng.random((20, 21))
    s = smooth(a)
    assert np.isclose(s.mean(), a.mean())
    s2 = smooth(a, restore_max=True)
    assert np.isclose(np.abs(s2).max(), np.abs(a).max())


def test_staggered_density():
    kg = KWaveGrid((4, 3), (1.0, 1.0))
    r = np.arange(12, dtype=float).reshape(4, 3) + 1
    sx, sy = staggered_density(r, kg)
    np.testing.assert_allclose(sx[:-1], 0.5 * (r[:-1] + r[1:]))
    np.testing.assert_array_equal(sx[-1], r[-1])  # outside the grid: original value
    np.testing.assert_allclose(sy[:, :-1], 0.5 * (r[:, :-1] + r[:, 1:]))


def test_source_scaling():
    """kspaceFirstOrder_scaleSourceTerms.m:50-128, 285-369."""
    n = (32, 32, 32)
    kg = KWaveGrid(n, (1e-4,) * 3)
    kg.set_time(10, 2e-8)
    mask = np.zeros(n)
    mask[5, 5:8, 6] = 1
    sig = np.ones((1, 10))
    med = {"sound_speed": 1500.0, "density": 1000.0}
    sens = {"mask": np.ones(n)}
    inp, _, _, _ = prepare(kg, med, {"p_mask": mask, "p": sig}, sens)
    assert np.allclose(inp["p_source_input"], 2 * 2e-8 / (3 * 1500.0 * 1e-4))
    assert inp["p_source_mode"] == 2 and inp["p_source_flag"] == 10
    inp, _, _, _ = prepare(kg, med, {"p_mask": mask, "p": sig, "p_mode": "dirichlet"}, sens)
    assert np.allclose(inp["p_source_input"], 1 / (3 * 1500.0 ** 2))
    inp, _, _, _ = prepare(kg, med, {"u_mask": mask, "ux": sig, "u_mode": "additive-no-correction"}, sens)
    assert np.allclose(inp["ux_source_input"], 2 * 1500.0 * 2e-8 / 1e-4) and inp["u_source_mode"] == 1


def test_time_reversal_becomes_dirichlet_source():
    n = (32, 32)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(20, 2e-8)
    mask = np.zeros(n)
    mask[3, :] = 1
    data = np.random.default_rng(1).random((32, 20))
    inp, record, _, meta = prepare(kg, {"sound_speed": 1500.0},
                                   {}, {"mask": mask, "time_reversal_boundary_data": data})
    assert meta["time_rev"] and record == ["p_final"] and inp["p_source_mode"] == 0
    np.testing.assert_allclose(inp["p_source_input"], np.fliplr(data) / (2 * 1500.0 ** 2))


def test_fourier_shift_half_sample():
    t = np.arange(64)
    x = np.sin(2 * np.pi * 3 * t / 64)
    y = fourier_shift(x, 0.5)
    np.testing.assert_allclose(y, np.sin(2 * np.pi * 3 * (t + 0.5) / 64), atol=1e-12)


def test_make_time_cfl():
    kg = KWaveGrid((100, 100), (1e-4, 2e-4))
    Nt, dt = kg.make_time(1500.0, 0.3)
    assert np.isclose(dt, 0.3 * 1e-4 / 1500)
    assert Nt == int(np.floor(np.hypot(1e-2, 2e-2) / 1500 / dt)) + 1
