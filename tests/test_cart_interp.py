"""Linear interpolation of Cartesian sensor points
(kspaceFirstOrder_extractSensorData.m:296-420 with the barycentric weights of
kspaceFirstOrder_createStorageVariables.m:372-394): weights, exactness on
linear fields, and the per-point reductions taken on interpolated series."""
import numpy as np
import pytest

from kwave.simulation import postprocess, prepare
from kwave.utils import KWaveGrid, cart_linear_weights, make_cart_circle, make_cart_sphere, make_disc


def _grid_coords(kg):
    """Coordinates of every grid point (column-major linear order)."""
    axes = [(np.arange(n) - n // 2) * d for n, d in zip(kg.N, kg.d)]
    mesh = np.meshgrid(*axes, indexing="ij")
    return np.stack([m.reshape(-1, order="F") for m in mesh])


@pytest.mark.parametrize("shape", [(20, 17), (12, 11, 10)])
def test_weights_are_barycentric_and_exact_for_linear_fields(shape):
    rng = np.random.default_rng(3)
    kg = KWaveGrid(shape, tuple(1e-4 * (1 + 0.1 * a) for a in range(len(shape))))
    lo = np.array([-(n // 2) * d for n, d in zip(kg.N, kg.d)])
    hi = np.array([(n - 1 - n // 2) * d for n, d in zip(kg.N, kg.d)])
    pts = lo[:, None] + rng.random((len(shape), 200)) * (hi - lo)[:, None]
    verts, w = cart_linear_weights(kg, pts)
    assert verts.shape == w.shape == (200, len(shape) + 1)
    assert np.all(w >= -1e-12) and np.allclose(w.sum(axis=1), 1.0)
    assert verts.min() >= 1 and verts.max() <= int(np.prod(shape))
    xyz = _grid_coords(kg)
    coef = rng.standard_normal(len(shape))
    field = 2.5 + coef @ xyz
    interp = np.sum(field[verts - 1] * w, axis=1)
    np.testing.assert_allclose(interp, 2.5 + coef @ pts, rtol=0, atol=1e-12)
    # each point lies in the simplex its vertices span: same coordinates back
    np.testing.assert_allclose(np.einsum("pj,apj->ap", w, xyz[:, verts - 1]), pts, rtol=0, atol=1e-15)


def test_grid_points_take_one_vertex():
    kg = KWaveGrid((16, 18, 14), (1e-4, 1e-4, 1e-4))
    idx = np.array([[0, 3, 15], [5, 17, 0], [7, 7, 13]])  # 0-based (x, y, z) per column
    pts = np.stack([(idx[a] - kg.N[a] // 2) * kg.d[a] for a in range(3)])
    verts, w = cart_linear_weights(kg, pts)
    lin = idx[0] + kg.N[0] * (idx[1] + kg.N[1] * idx[2]) + 1
    for j in range(3):
        keep = w[j] > 1e-12
        assert keep.sum() == 1 and verts[j][keep][0] == lin[j]


def test_points_outside_the_grid_are_rejected():
    kg = KWaveGrid((16, 16), (1e-4, 1e-4))
    with pytest.raises(ValueError):
        cart_linear_weights(kg, np.array([[0.0], [8.5e-4]]))


def test_linear_sensor_outputs_through_the_oracle():
    """The point outputs are the weighted vertex sums each step, and max /
    min / rms are reductions of those series: checked against a run that
    records the vertices themselves as a binary mask."""
    from oracle.kspace_oracle import simulate

    n = (48, 40)
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(60, 0.3 * 1e-4 / 1500)
    p0 = 2 * make_disc(n[0], n[1], 24, 20, 4)
    pts = make_cart_circle(1.3e-3, 9)
    rec = ["p", "p_max", "p_min", "p_rms", "u_max", "u_rms"]
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    inp, record, start, meta = prepare(kg, medium, {"p0": p0}, {"mask": pts, "record": rec}, pml_size=6,
                                       cart_interp="linear")
    assert record == rec and inp["sensor_interp_index"].shape == (9, 3)
    out = postprocess(simulate(inp, record=record, record_start_index=start, dtype=np.float64), inp, meta)
    assert set(out) == {"p", "p_max", "p_min", "p_rms", "ux_max", "uy_max", "ux_rms", "uy_rms"}
    verts, w = inp["sensor_interp_index"], inp["sensor_interp_weight"]
    uniq = np.unique(verts)
    vin = dict(inp, sensor_mask_index=uniq)
    vin.pop("sensor_interp_index")
    vin.pop("sensor_interp_weight")
    raw = simulate(vin, record=["p", "u"], dtype=np.float64)
    col = np.searchsorted(uniq, verts)
    p = np.einsum("pj,pjt->pt", w, raw["p"][col])
    np.testing.assert_allclose(out["p"], p, rtol=1e-12, atol=1e-12 * np.abs(p).max())
    np.testing.assert_allclose(out["p_max"], p.max(axis=1), rtol=1e-12)
    np.testing.assert_allclose(out["p_min"], p.min(axis=1), rtol=1e-12)
    np.testing.assert_allclose(out["p_rms"], np.sqrt(np.mean(p * p, axis=1)), rtol=1e-10)
    uy = np.einsum("pj,pjt->pt", w, raw["uy"][col])
    np.testing.assert_allclose(out["uy_max"], uy.max(axis=1), rtol=1e-12)
    # against nearest-point recording of the same circle: same field, close values
    inp_n, record_n, _, meta_n = prepare(kg, medium, {"p0": p0}, {"mask": pts, "record": ["p"]}, pml_size=6)
    near = postprocess(simulate(inp_n, record=record_n, dtype=np.float64), inp_n, meta_n)
    assert np.max(np.abs(near["p"] - out["p"])) < 0.5 * np.abs(near["p"]).max()


def test_linear_interp_inputs_and_file_refusal(tmp_path):
    from kwave import h5io

    kg = KWaveGrid((24, 24, 24), (1e-4, 1e-4, 1e-4))
    kg.set_time(10, 1e-8)
    pts = make_cart_sphere(8e-4, 30)
    inp, record, _, meta = prepare(kg, {"sound_speed": 1500.0}, {"p0": np.zeros(kg.N)},
                                   {"mask": pts, "record": ["p"]}, pml_size=4, cart_interp="linear")
    v, w = cart_linear_weights(kg, pts)
    np.testing.assert_array_equal(inp["sensor_interp_index"], v)
    np.testing.assert_allclose(inp["sensor_interp_weight"], w)
    assert "sensor_mask_index" not in inp
    with pytest.raises(ValueError, match="interpolated"):
        h5io.write_input_file(tmp_path / "x.h5", inp)
    with pytest.raises(ValueError):
        prepare(kg, {"sound_speed": 1500.0}, {"p0": np.zeros(kg.N)}, {"mask": pts}, cart_interp="cubic")
