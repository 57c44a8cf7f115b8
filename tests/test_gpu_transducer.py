"""Transducer source and sensor on the GPU (kspaceFirstOrder3D.m:886-902;
kspaceFirstOrder3DC.m:780-783): the CUDA path against the FP64 oracle at the
lossless bar, against the equivalent per-point velocity source, and through
the input file."""
import numpy as np
import pytest

from helpers import oracle_outputs, rel_l2

pytestmark = pytest.mark.gpu

TOL_LOSSLESS = 1e-5


def _case(elev=True, apod="Hanning", nt=70):
    from kwave.simulation import prepare
    from kwave.transducer import KWaveTransducer
    from kwave.utils import KWaveGrid, tone_burst

    kg = KWaveGrid((40, 48, 32), (1e-4, 1e-4, 1e-4))
    kg.set_time(nt, 0.3e-4 / 1500)
    sig = tone_burst(1 / kg.dt, 2.5e6, 2).ravel()
    tr = KWaveTransducer(kg, number_elements=7, element_width=2, element_length=6, element_spacing=1,
                         position=(8, 10, 12), steering_angle=12, focus_distance=2e-3, sound_speed=1500.0,
                         elevation_focus_distance=1.5e-3 if elev else np.inf, transmit_apodization=apod,
                         input_signal=sig)
    mask = np.zeros(kg.N)
    mask[20, 8:40:3, 6:26:4] = 1
    sensor = {"mask": mask, "record": ["p", "p_max", "u", "p_final"]}
    return prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, tr, sensor, pml_size=6), kg


def test_transducer_source_matches_oracle():
    from kwave import _lib

    (inp, record, start, meta), _ = _case()
    assert inp["transducer_source_flag"] > 0 and "transducer_source_apodization" in inp
    gpu = _lib.solve(inp, record=record, start_index=start)
    ora = oracle_outputs(inp, record, start, dtype=np.float64)
    errs = {k: rel_l2(gpu[k], ora[k]) for k in ("p", "p_max", "ux", "uy", "uz", "p_final")}
    assert max(errs.values()) <= TOL_LOSSLESS, errs
    assert np.abs(ora["p"]).max() > 0


def test_transducer_source_equals_velocity_source():
    """Same field as an additive-no-correction x-velocity source with one
    signal per point (input sample delay + t - 1, times the apodization)."""
    from kwave import _lib

    (inp, record, start, meta), _ = _case()
    flag = inp["transducer_source_flag"]
    rows = (inp["delay_mask"] - 1)[:, None] + np.arange(flag)[None, :]
    sig32 = np.asarray(inp["transducer_source_input"], np.float32)
    apod32 = np.asarray(inp["transducer_source_apodization"], np.float32)
    eq = {k: v for k, v in inp.items() if not k.startswith("transducer") and k != "delay_mask"}
    eq.update(ux_source_flag=flag, u_source_mode=1, u_source_many=1,
              ux_source_input=(apod32[:, None] * sig32[rows]).astype(np.float32))
    a = _lib.solve(inp, record=record, start_index=start)
    b = _lib.solve(eq, record=record, start_index=start)
    for k in ("p", "ux", "p_final"):
        assert rel_l2(a[k], b[k]) <= 1e-6, k


def test_transducer_input_file_matches_solve(tmp_path):
    from kwave import _lib, h5io

    (inp, record, start, meta), _ = _case(apod="Rectangular")
    assert "transducer_source_apodization" not in inp
    fin, fout = tmp_path / "in.h5", tmp_path / "out.h5"
    h5io.write_input_file(fin, inp)
    _lib.run_file(fin, fout, record)
    got = h5io.read_output_file(fout, 3)
    want = _lib.solve(inp, record=record)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_transducer_as_sensor():
    """A transducer records pressure at its active grid points; the series
    come back averaged per element, GPU and oracle through the same
    postprocess()."""
    from kwave import _lib
    from kwave.simulation import postprocess, prepare
    from kwave.transducer import KWaveTransducer
    from kwave.utils import KWaveGrid, make_ball

    kg = KWaveGrid((36, 40, 30), (1e-4, 1e-4, 1e-4))
    kg.set_time(60, 0.3e-4 / 1500)
    tr = KWaveTransducer(kg, number_elements=6, element_width=2, element_length=5, element_spacing=1,
                         position=(6, 8, 10), elevation_focus_distance=1e-3, sound_speed=1500.0)
    p0 = 3 * make_ball(*kg.N, 24, 20, 14, 3)
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": p0}, tr,
                                       pml_size=6)
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(oracle_outputs(inp, record, start, dtype=np.float64), inp, meta)
    assert gpu.shape == (6, 60)
    assert rel_l2(gpu, ora) <= TOL_LOSSLESS
