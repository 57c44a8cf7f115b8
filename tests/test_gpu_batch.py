"""Batches (kw_batch_*): sessions advanced together, one CUDA graph launch per
time step for all of them, give bit for bit the outputs of each session run
alone -- across grids, dimensions, Nt, initial-pressure starts, slab chains
on two streams and chunked advancing."""
import os

import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het

pytestmark = pytest.mark.gpu


def _cases():
    from kwave import _lib

    _lib.wisdom_forget()  # built-in schedules throughout
    a = case_2d_p0(n=(64, 48), nt=37)
    b = case_3d_het(n=(64, 48, 40), nt=30, record=("p", "p_max", "p_rms", "u", "p_final"))
    c = case_3d_het(n=(72, 64, 30), nt=23, absorbing=False, nonlinear=False, record=("p", "p_final"))
    return [a, b, c]


def _alone(case):
    from kwave import _lib

    inp, record, start, _ = case
    s = _lib.Session(inp, record, start)
    s.advance(int(inp["Nt"]))
    out = s.read()
    s.close()
    return out


@pytest.mark.parametrize("chunk", [1, 7, 1000])
def test_batch_matches_sessions_alone(chunk):
    from kwave import _lib

    cases = _cases()
    ref = [_alone(c) for c in cases]
    sessions = [_lib.Session(inp, record, start) for inp, record, start, _ in cases]
    b = _lib.Batch(sessions)
    nt_max = max(int(c[0]["Nt"]) for c in cases)
    for _ in range(0, nt_max, chunk):
        b.advance(chunk)
    b.sync()
    launches = b.graph_launches
    b.close()
    assert all(s.steps_done == int(c[0]["Nt"]) for s, c in zip(sessions, cases))
    # every step but the first (initial pressure / graph capture) and the last
    # of the longest run is one parent-graph launch
    assert nt_max - 2 <= launches <= nt_max
    for s, r in zip(sessions, ref):
        out = s.read()
        s.close()
        for k in r:
            np.testing.assert_array_equal(out[k], r[k], err_msg=k)


def test_batch_with_slab_chains_on_two_streams():
    from kwave import _lib

    _lib.wisdom_forget()
    case = case_3d_het(n=(64, 48, 40), nt=21, record=("p", "p_max", "u"))
    ref = _alone(case)
    inp, record, start, _ = case
    old = {k: os.environ.get(k) for k in ("KWAVE_B200_SLAB", "KWAVE_B200_SLAB_STREAMS")}
    os.environ.update(KWAVE_B200_SLAB="20", KWAVE_B200_SLAB_STREAMS="2")
    try:
        sessions = [_lib.Session(inp, record, start) for _ in range(2)]
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    assert sessions[0].schedule["streams"] == 2
    b = _lib.Batch(sessions)
    b.advance(int(inp["Nt"]))
    ms = b.elapsed_ms()
    assert ms > 0
    b.close()
    for s in sessions:
        out = s.read()
        s.close()
        for k in ref:
            np.testing.assert_array_equal(out[k], ref[k], err_msg=k)


def test_run_batch_graph_mode_and_bad_batches():
    from kwave import _lib, serving

    cases = _cases()
    inputs = [c[0] for c in cases]
    outs_g = serving.run_batch(inputs, record=("p",), chunk=10, mode="graph")
    outs_s = serving.run_batch(inputs, record=("p",), chunk=10, mode="streams")
    for a, b in zip(outs_g, outs_s):
        np.testing.assert_array_equal(a["p"], b["p"])
    s = _lib.Session(inputs[0], ("p",))
    with pytest.raises(_lib.KwaveError, match="twice"):
        _lib.Batch([s, s])
    s.close()
    with pytest.raises(ValueError):
        serving.run_batch(inputs[:1], mode="bogus")
