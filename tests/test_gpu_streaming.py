"""Streamed raw series: when the recorded time series would exceed the
recording budget, kw_solve keeps only a ring of steps on the device and
drains it to the host in blocks.  The outputs are the same, bit for bit, as
with the whole series held on the device."""
import os

import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het

pytestmark = pytest.mark.gpu


def _solve_with_budget(inp, record, start, budget):
    from kwave import _lib

    old = os.environ.get("KWAVE_B200_RECORD_BUDGET")
    os.environ["KWAVE_B200_RECORD_BUDGET"] = str(budget)
    try:
        return _lib.solve(inp, record, start_index=start)
    finally:
        if old is None:
            del os.environ["KWAVE_B200_RECORD_BUDGET"]
        else:
            os.environ["KWAVE_B200_RECORD_BUDGET"] = old


def _same(a, b):
    assert set(a) == set(b)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("rows", [1, 7, 23])
def test_streamed_series_2d(rows):
    from kwave import _lib

    record = ("p", "u", "u_non_staggered", "p_max", "p_final")
    inp, _, _, _ = case_2d_p0(n=(64, 48), nt=50, record=record)
    full = _lib.solve(inp, record, start_index=5)
    ns = full["p"].shape[0]
    per_step = 4 * ns * (1 + 2 + 2)  # p, ux, uy, ux/uy on the regular grid
    streamed = _solve_with_budget(inp, record, 5, per_step * rows + 1)
    _same(streamed, full)


def test_streamed_series_3d_source():
    from kwave import _lib

    record = ("p", "u", "p_rms")
    inp, _, _, _ = case_3d_het(n=(36, 30, 32), nt=40, record=record)
    full = _lib.solve(inp, record)
    ns = full["p"].shape[0]
    streamed = _solve_with_budget(inp, record, 1, 4 * ns * 4 * 9 + 1)  # a ring of 9 steps
    _same(streamed, full)


def test_streamed_interpolated_points():
    """Cartesian points interpolated on the device stream like grid points."""
    from kwave import _lib
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_cart_circle, make_disc

    kg = KWaveGrid((64, 64), (1e-4, 1e-4))
    kg.set_time(60, 0.3e-4 / 1500)
    record = ["p", "u", "u_non_staggered", "p_max"]
    inp, record, start, _ = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0},
                                    {"p0": 2 * make_disc(64, 64, 32, 30, 4)},
                                    {"mask": make_cart_circle(2e-3, 20), "record": record}, pml_size=8,
                                    cart_interp="linear")
    full = _lib.solve(inp, record, start_index=3)
    streamed = _solve_with_budget(inp, record, 3, 4 * 20 * 5 * 6 + 1)  # a ring of 6 steps
    _same(streamed, full)
