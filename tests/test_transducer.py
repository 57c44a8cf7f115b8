"""Linear-array transducer (kWaveTransducer.m) and its source / sensor
branches: geometry, beamforming delays, padded input signal, the source
datasets (kspaceFirstOrder_inputChecking.m:1155-1213) and the loop term
(kspaceFirstOrder3D.m:886-902) in the oracle, the per-element combine
(kWaveTransducer.m:907-950) and the file-path handling."""
import warnings

import numpy as np
import pytest

from kwave.simulation import postprocess, prepare
from kwave.transducer import KWaveTransducer
from kwave.utils import KWaveGrid, get_win_1d, tone_burst


def _grid(n=(24, 40, 24), nt=40):
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(nt, 0.3e-4 / 1500)
    return kg


def test_geometry_and_masks():
    kg = _grid()
    tr = KWaveTransducer(kg, number_elements=6, element_width=2, element_length=5, element_spacing=1,
                         position=(4, 3, 8), active_elements=[0, 1, 1, 1, 0, 1])
    assert tr.transducer_width == 6 * 2 + 5
    im = tr.indexed_elements_mask
    assert set(np.unique(im)) == set(range(7)) and np.count_nonzero(im) == 6 * 2 * 5
    assert np.all(im[3, 2:4, 7:12] == 1) and np.all(im[3, 5:7, 7:12] == 2) and im[3, 4, 7] == 0
    assert tr.number_active_elements == 4
    assert tr.active_elements_mask.sum() == 4 * 10 and np.all(tr.active_elements_mask[3, 2:4] == 0)
    ia = tr.indexed_active_elements_mask  # lowest active element becomes 1; gaps are kept
    assert ia[3, 5, 7] == 1 and ia[3, 11, 7] == 3 and ia[3, 17, 7] == 5 and ia[3, 2, 7] == 0 and ia[3, 14, 7] == 0
    assert np.all(tr.indexed_element_voxel_mask[3, 2, 7:12] == np.arange(1, 6))
    with pytest.raises(ValueError, match="y-direction"):
        KWaveTransducer(kg, number_elements=20, element_width=2, position=(4, 3, 8), element_length=5)
    with pytest.raises(ValueError, match="radius"):
        KWaveTransducer(kg, number_elements=2, element_length=5, position=(1, 1, 1), radius=0.1)


def test_steered_and_focussed_delays():
    kg = _grid()
    c = 1540.0
    tr = KWaveTransducer(kg, number_elements=8, element_width=2, element_length=4, position=(3, 4, 6),
                         steering_angle=20, sound_speed=c)
    pitch = 2 * kg.dy
    idx = np.arange(8) - 3.5
    t = pitch * idx * np.sin(np.deg2rad(20)) / c / kg.dt
    expect = np.sign(t) * np.floor(np.abs(t) + 0.5)
    np.testing.assert_array_equal(tr.beamforming_delays(), expect)
    dm = tr.delay_mask()
    per_el = np.array([dm[2, 3 + 2 * e, 5] for e in range(8)])
    np.testing.assert_array_equal(per_el, -expect - (-expect).min())
    assert dm.min() == 0 and np.count_nonzero(dm) <= 8 * 2 * 4
    # a focus: symmetric delays, largest at the centre
    trf = KWaveTransducer(kg, number_elements=8, element_width=2, element_length=4, position=(3, 4, 6),
                          focus_distance=2e-3, elevation_focus_distance=1.5e-3, sound_speed=c)
    bd = trf.beamforming_delays()
    np.testing.assert_array_equal(bd, bd[::-1])
    ed = trf.elevation_beamforming_delays()
    np.testing.assert_array_equal(ed, ed[::-1])
    assert ed[0] >= ed[1] >= 0 and ed[-1] >= 0
    dm2 = trf.delay_mask(2)  # elevation only: constant along each element's y extent
    assert np.all(dm2[2, 4, 5:9] == dm2[2, 5, 5:9])


def test_input_signal_padding_and_steering_max():
    kg = _grid()
    sig = np.r_[0.0, 1.0, 2.0, 1.0, 0.0]
    tr = KWaveTransducer(kg, number_elements=8, element_width=2, element_length=4, position=(3, 4, 6),
                         steering_angle=30, input_signal=sig)
    dmax = int(tr.delay_mask().max())
    padded = tr.input_signal
    assert padded.size == sig.size + 2 * dmax  # one zero each side already
    assert np.flatnonzero(padded)[0] == dmax + 1 and padded.size - 1 - np.flatnonzero(padded)[-1] == dmax + 1
    trm = KWaveTransducer(kg, number_elements=8, element_width=2, element_length=4, position=(3, 4, 6),
                          steering_angle_max=30, steering_angle=10, input_signal=sig)
    bd = -tr.beamforming_delays()  # the delays at the maximum angle fix the padding
    assert trm.appended_zeros == bd.max() - bd.min() and trm.beamforming_delays_offset == -bd.min()
    assert trm.input_signal.size == sig.size + 2 * trm.appended_zeros
    dm = trm.delay_mask()
    assert dm[trm.active_elements_mask != 0].min() >= 0
    with pytest.raises(ValueError):
        trm.steering_angle = 40


def test_apodization_windows():
    kg = _grid()
    tr = KWaveTransducer(kg, number_elements=6, element_width=2, element_length=3, position=(3, 4, 6),
                         transmit_apodization="Hanning")
    m = tr.transmit_apodization_mask()
    w = get_win_1d(6, "Hanning")
    np.testing.assert_allclose([m[2, 3 + 2 * e, 5] for e in range(6)], w)
    assert np.count_nonzero(m) == np.count_nonzero(w) * 2 * 3


def test_source_datasets_and_oracle_equivalence():
    """The transducer term equals an additive-no-correction x-velocity source
    with one signal per point: row i = apodization_i * input(delay_i + t - 1)."""
    from oracle.kspace_oracle import simulate

    kg = _grid(n=(24, 32, 20), nt=50)
    sig = tone_burst(1 / kg.dt, 3e6, 2)
    tr = KWaveTransducer(kg, number_elements=5, element_width=2, element_length=4, element_spacing=1,
                         position=(6, 5, 8), steering_angle=15, transmit_apodization="Hanning",
                         input_signal=sig.ravel())
    sensor = {"mask": np.pad(np.ones((1, 4, 4)), ((14, 9), (14, 14), (8, 8))), "record": ["p", "u"]}
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    inp, record, start, meta = prepare(kg, medium, tr, sensor, pml_size=4)
    n = int(tr.active_elements_mask.sum())
    assert inp["u_source_index"].size == n and inp["delay_mask"].min() >= 1
    flag = inp["transducer_source_flag"]
    padded = tr.input_signal * (2 * 1500.0 * kg.dt / kg.dx)
    assert flag == padded.size - tr.delay_mask().max()
    np.testing.assert_allclose(inp["transducer_source_input"], padded)
    apod = inp["transducer_source_apodization"]
    eq = {k: v for k, v in inp.items() if not k.startswith("transducer") and k != "delay_mask"}
    rows = (inp["delay_mask"] - 1)[:, None] + np.arange(flag)[None, :]
    eq.update(ux_source_flag=flag, u_source_mode=1, u_source_many=1,
              ux_source_input=apod[:, None] * inp["transducer_source_input"][rows])
    a = simulate(inp, record=record, dtype=np.float64)
    b = simulate(eq, record=record, dtype=np.float64)
    for k in ("p", "ux", "uy", "uz"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-12, atol=1e-12 * np.abs(b[k]).max())
    assert np.abs(a["p"]).max() > 0


def test_transducer_sensor_combines_per_element():
    kg = _grid(n=(16, 24, 16), nt=12)
    tr = KWaveTransducer(kg, number_elements=4, element_width=2, element_length=3, element_spacing=1,
                         position=(5, 3, 6), active_elements=[1, 1, 0, 1])
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0}, {"p0": np.zeros(kg.N)}, tr, pml_size=4)
    assert record == ["p"] and inp["sensor_mask_index"].size == 3 * 6
    ia = tr.indexed_active_elements_mask.reshape(-1, order="F")
    el = ia[ia > 0]
    series = el[:, None] * np.ones((1, 12)) + np.arange(12)[None, :]
    out = postprocess({"p": series.copy()}, inp, meta)
    # element indices keep the gap of the inactive element: a zero third row
    assert out.shape == (4, 12)
    for r in (0, 1, 3):
        np.testing.assert_allclose(out[r], (r + 1) + np.arange(12))
    assert not out[2].any()
    # with an elevation focus each point's series is advanced by its delay
    trf = KWaveTransducer(kg, number_elements=2, element_width=1, element_length=5, position=(5, 3, 6),
                          elevation_focus_distance=1e-3)
    dm = trf.delay_mask(2).reshape(-1, order="F")[trf.active_elements_mask.reshape(-1, order="F") != 0]
    data = np.tile(np.arange(12.0), (10, 1))
    comb = trf.combine_sensor_data(data)
    expect = np.zeros(12)
    for d in dm[:5]:
        expect[:12 - d] += np.arange(12.0)[d:]
    np.testing.assert_allclose(comb[0], expect / 5)


def test_scan_line_delay_and_sum():
    kg = _grid()
    tr = KWaveTransducer(kg, number_elements=4, element_width=2, element_length=3, position=(3, 4, 6),
                         steering_angle=25)
    d = -tr.beamforming_delays()
    data = np.zeros((4, 30))
    for e in range(4):
        data[e, 10 + d[e]] = 1.0  # an echo arriving with the element's delay
    line = tr.scan_line(data)
    assert line[10] == 4.0


def test_file_path_datasets(tmp_path):
    import torch

    from kwave import _lib, h5io

    kg = _grid(n=(16, 24, 16), nt=20)
    tr = KWaveTransducer(kg, number_elements=3, element_width=2, element_length=3, position=(5, 3, 6),
                         steering_angle=10, input_signal=np.r_[0, 1.0, -1.0, 0.5], transmit_apodization="Hanning")
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0}, tr, {"mask": np.ones(kg.N)}, pml_size=4)
    f = tmp_path / "tr.h5"
    with pytest.warns(UserWarning, match="apodization"):
        h5io.write_input_file(f, inp)
    F = h5io.File(f)
    np.testing.assert_array_equal(F.read("/delay_mask").reshape(-1), inp["delay_mask"])
    assert int(F.read("/transducer_source_flag").reshape(-1)[0]) == inp["transducer_source_flag"]
    np.testing.assert_allclose(F.read("/transducer_source_input").reshape(-1),
                               np.asarray(inp["transducer_source_input"], np.float32))
    if not torch.cuda.is_available():
        try:
            _lib.run_file(f, tmp_path / "o.h5", record)
            code = 0
        except _lib.KwaveError as e:
            code = e.code
        assert code == _lib.KW_ERR_CUDA  # the whole file was read
    bad = dict(inp, delay_mask=inp["delay_mask"][:-1])
    bad.pop("transducer_source_apodization")
    h5io.write_input_file(tmp_path / "bad.h5", bad)
    with pytest.raises(_lib.KwaveError) as e:
        _lib.run_file(tmp_path / "bad.h5", tmp_path / "o.h5", record)
    assert e.value.code == _lib.KW_ERR_IO and "delay_mask" in str(e.value)


def test_one_array_transmits_and_receives():
    kg = _grid(n=(16, 24, 16), nt=12)
    tr = KWaveTransducer(kg, number_elements=3, element_width=2, element_length=3, position=(5, 3, 6),
                         input_signal=np.r_[0, 1.0, 0])
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0}, tr, tr, pml_size=4)
    np.testing.assert_array_equal(inp["u_source_index"], inp["sensor_mask_index"])
    assert record == ["p"] and meta["transducer"] is tr and inp["transducer_source_flag"] == 3
