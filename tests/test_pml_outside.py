"""PMLInside = false (kspaceFirstOrder_expandGridMatrices.m;
kspaceFirstOrder3DC.m:586-614): the grid grows by the PML on every side,
the inputs follow, and the full-grid outputs are cut back to the user's grid."""
import numpy as np
import pytest

from kwave.simulation import postprocess, prepare
from kwave.transducer import KWaveTransducer
from kwave.utils import KWaveGrid, make_cart_circle, make_disc, smooth


def test_expanded_inputs():
    n, P = (30, 26), (5, 7)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(20, 2e-8)
    rng = np.random.default_rng(0)
    c = 1500 + 20 * rng.random(n)
    p0 = make_disc(*n, 15, 13, 4)
    mask = np.zeros(n)
    mask[3, 4] = mask[20, 2] = 1
    inp, record, start, meta = prepare(kg, {"sound_speed": c, "density": 1000.0}, {"p0": p0},
                                       {"mask": mask, "record": ["p", "p_final"]}, pml_size=P, pml_inside=False)
    N = (n[0] + 2 * P[0], n[1] + 2 * P[1])
    assert (inp["Nx"], inp["Ny"]) == N and inp["Nt"] == 20 and inp["dt"] == 2e-8
    np.testing.assert_array_equal(np.asarray(inp["c0"]).reshape(N, order="F") if np.size(inp["c0"]) > 1 else 0,
                                  np.pad(c, [(5, 5), (7, 7)], mode="edge"))
    np.testing.assert_allclose(np.asarray(inp["p0_source_input"]).reshape(N),
                               np.pad(smooth(p0, True), [(5, 5), (7, 7)]))
    lin = np.flatnonzero(np.pad(mask, [(5, 5), (7, 7)]).reshape(-1, order="F")) + 1
    np.testing.assert_array_equal(inp["sensor_mask_index"], lin)
    out = postprocess({"p": np.zeros((2, 20), np.float32), "p_final": np.arange(np.prod(N)).reshape(N)},
                      inp, meta)
    assert out["p_final"].shape == n and out["p_final"][0, 0] == 5 * N[1] + 7


def test_cuboid_and_cartesian_sensors_shift():
    n, P = (24, 20, 18), 4
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(10, 2e-8)
    corners = np.array([[3, 4, 5, 8, 9, 7]]).T
    inp, _, _, meta = prepare(kg, {"sound_speed": 1500.0}, {"p0": np.zeros(n)}, {"mask": corners},
                              pml_size=P, pml_inside=False)
    np.testing.assert_array_equal(inp["sensor_mask_corners"], corners + P)
    kg2 = KWaveGrid(n[:2], (1e-4, 1e-4))
    kg2.set_time(10, 2e-8)
    pts = make_cart_circle(6e-4, 7)
    a, _, _, _ = prepare(kg2, {"sound_speed": 1500.0}, {"p0": np.zeros(n[:2])}, {"mask": pts}, pml_size=P)
    b, _, _, _ = prepare(kg2, {"sound_speed": 1500.0}, {"p0": np.zeros(n[:2])}, {"mask": pts}, pml_size=P,
                         pml_inside=False)
    ia = np.asarray(a["sensor_mask_index"]) - 1
    x, y = ia % n[0], ia // n[0]
    np.testing.assert_array_equal(np.asarray(b["sensor_mask_index"]) - 1, (x + P) + (n[0] + 2 * P) * (y + P))


def test_transducer_expands_without_changing_the_user_object():
    n = (16, 24, 16)
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(12, 2e-8)
    tr = KWaveTransducer(kg, number_elements=3, element_width=2, element_length=3, position=(5, 3, 6),
                         steering_angle=10, input_signal=np.r_[0, 1.0, -1.0, 0])
    a, _, _, _ = prepare(kg, {"sound_speed": 1500.0}, tr, tr, pml_size=4)
    b, _, _, meta = prepare(kg, {"sound_speed": 1500.0}, tr, tr, pml_size=4, pml_inside=False)
    assert tr.stored_grid_size == n and meta["transducer"].stored_grid_size == (24, 32, 24)
    np.testing.assert_array_equal(a["delay_mask"], b["delay_mask"])
    np.testing.assert_array_equal(b["u_source_index"], b["sensor_mask_index"])
    ia = np.asarray(a["u_source_index"]) - 1
    x, y, z = ia % 16, (ia // 16) % 24, ia // (16 * 24)
    np.testing.assert_array_equal(np.asarray(b["u_source_index"]) - 1, (x + 4) + 24 * ((y + 4) + 32 * (z + 4)))


def test_outside_pml_agrees_with_free_space_before_the_wave_arrives():
    """Before the wave reaches the edge of the user's grid, an inside and an
    outside PML see the same free-space field."""
    from oracle.kspace_oracle import simulate

    n = (64, 64)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(40, 0.3e-4 / 1500)
    p0 = 2 * make_disc(*n, 32, 32, 4)
    rec = {"mask": np.ones(n), "record": ["p_final"]}
    out = {}
    for inside in (True, False):
        inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": p0}, rec,
                                           pml_size=10, pml_inside=inside)
        res = simulate(inp, record=record, dtype=np.float64)
        out[inside] = postprocess(res, inp, meta)["p_final"]
    assert out[False].shape == n
    core = (slice(14, 50), slice(14, 50))
    err = np.linalg.norm(out[True][core] - out[False][core]) / np.linalg.norm(out[False][core])
    assert err < 2e-3, err


def test_axisymmetric_grid_grows_at_the_outer_radius_only():
    n, P = (40, 20), (6, 5)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(20, 2e-8)
    mask = np.zeros(n)
    mask[10, 0] = mask[30, 7] = 1
    inp, record, _, meta = prepare(kg, {"sound_speed": 1500.0}, {"p0": make_disc(*n, 20, 1, 4)},
                                   {"mask": mask, "record": ["p", "p_final"]}, pml_size=P, pml_inside=False,
                                   axisymmetric=True)
    assert (inp["Nx"], inp["Ny"]) == (52, 25) and inp["axisymmetric_flag"] == 1
    lin = np.flatnonzero(np.pad(mask, [(6, 6), (0, 5)]).reshape(-1, order="F")) + 1
    np.testing.assert_array_equal(inp["sensor_mask_index"], lin)
    out = postprocess({"p": np.zeros((2, 20), np.float32), "p_final": np.arange(52 * 25).reshape(52, 25)}, inp, meta)
    assert out["p_final"].shape == n and out["p_final"][0, 0] == 6 * 25
