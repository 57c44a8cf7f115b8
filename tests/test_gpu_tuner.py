"""Launch-schedule tuner (kw_tune) and wisdom: every schedule it can pick
gives bit-identical outputs, sessions pick up what was tuned or imported,
and a tuned choice is written to and read back from a wisdom file."""
import os

import numpy as np
import pytest

from helpers import case_3d_het

pytestmark = pytest.mark.gpu

RECORD = ("p", "p_max", "p_rms", "u", "p_final")


class _env:
    """Set environment variables for the duration of a block."""

    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        for k, v in self.kv.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _schedule_of(inp, record=RECORD):
    from kwave import _lib

    s = _lib.Session(inp, record)
    try:
        return s.schedule
    finally:
        s.close()


def _forced(tmp_path, inp, **fields):
    """Tune once (to learn the key), then import a wisdom entry with the
    given schedule fields for that key."""
    from kwave import _lib

    _lib.wisdom_forget()
    _lib.tune(inp, RECORD)
    path = str(tmp_path / "w.txt")
    _lib.wisdom_export(path)
    lines = [l for l in open(path) if not l.startswith("#")]
    assert len(lines) == 1
    key, slab, streams, rows, cols, radix, ms = lines[0].split()
    vals = {"slab_planes": slab, "streams": streams, "row_lines": rows, "col_lines": cols, "radix_plan": radix}
    vals.update({k: str(v) for k, v in fields.items()})
    with open(path, "w") as f:
        f.write(f"{key} {vals['slab_planes']} {vals['streams']} {vals['row_lines']} {vals['col_lines']} "
                f"{vals['radix_plan']} {ms}\n")
    _lib.wisdom_forget()
    _lib.wisdom_import(path)


def test_tune_times_candidates_and_sessions_use_the_choice():
    from kwave import _lib

    inp, record, start, _ = case_3d_het(n=(64, 48, 40), nt=20, record=RECORD)
    _lib.wisdom_forget()
    default = _schedule_of(inp)
    assert default["slab_planes"] == 40 and default["streams"] == 1
    r = _lib.tune(inp, RECORD)
    assert r["candidates"] >= 4
    assert r["ms_per_step"] > 0 and r["ms_default"] > 0
    got = _schedule_of(inp)
    for k in ("slab_planes", "streams", "row_lines", "col_lines", "radix_plan"):
        assert got[k] == r[k], k
    _lib.wisdom_forget()
    assert _schedule_of(inp) == default


@pytest.mark.parametrize("slab,streams", [(14, 2), (20, 1), (10, 2)])
def test_every_slab_schedule_gives_identical_results(tmp_path, slab, streams):
    from kwave import _lib

    inp, record, start, _ = case_3d_het(n=(64, 48, 40), nt=30, record=RECORD)
    _lib.wisdom_forget()
    whole = _lib.solve(inp, RECORD, start_index=start)
    _forced(tmp_path, inp, slab_planes=slab, streams=streams, radix_plan=0)
    sc = _schedule_of(inp)
    assert (sc["slab_planes"], sc["streams"]) == (slab, streams)
    split = _lib.solve(inp, RECORD, start_index=start)
    _lib.wisdom_forget()
    for k in whole:
        np.testing.assert_array_equal(split[k], whole[k], err_msg=k)


def test_runtime_engine_tiles_give_identical_results(tmp_path):
    """x = 70 and y = 56 (factor 7) run on the runtime-plan engine, whose row
    and column tiles the tuner may halve."""
    from kwave import _lib

    inp, record, start, _ = case_3d_het(n=(70, 56, 32), nt=24, record=RECORD)
    _lib.wisdom_forget()
    base = _lib.solve(inp, RECORD, start_index=start)
    d = _schedule_of(inp)
    r = _lib.tune(inp, RECORD)
    assert r["candidates"] >= 2
    _forced(tmp_path, inp, row_lines=max(1, d["row_lines"] // 2), col_lines=4, radix_plan=0)
    sc = _schedule_of(inp)
    assert sc["row_lines"] == max(1, d["row_lines"] // 2) and sc["col_lines"] == 4
    tiled = _lib.solve(inp, RECORD, start_index=start)
    _lib.wisdom_forget()
    for k in base:
        np.testing.assert_array_equal(tiled[k], base[k], err_msg=k)


def test_wisdom_file_from_env_and_auto_tuning(tmp_path):
    """KWAVE_B200_TUNE=1: a session tunes itself on a miss and the choice is
    merged into the KWAVE_B200_WISDOM file; a process that forgot everything
    reads it back from the file."""
    from kwave import _lib

    inp, record, start, _ = case_3d_het(n=(64, 48, 40), nt=20, record=RECORD)
    path = str(tmp_path / "wisdom.txt")
    _lib.wisdom_forget()
    ref = _lib.solve(inp, RECORD, start_index=start)
    with _env(KWAVE_B200_TUNE="1", KWAVE_B200_WISDOM=path):
        out = _lib.solve(inp, RECORD, start_index=start)
    assert os.path.exists(path)
    entries = [l.split() for l in open(path) if not l.startswith("#")]
    assert len(entries) == 1 and entries[0][0].startswith("64x48x40/")
    if entries[0][5] == "0":  # the default radix order: only launch shapes differ
        for k in ref:
            np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
    else:  # y = 48 and z = 40 run on the runtime engine, whose radix order rounds differently
        from helpers import compare

        errs = compare(out, ref)
        assert max(errs.values()) <= 1e-5, errs
    _lib.wisdom_forget()
    _lib.wisdom_import(path)
    sc = _schedule_of(inp)
    assert (sc["slab_planes"], sc["streams"]) == (int(entries[0][1]), int(entries[0][2]))
    _lib.wisdom_forget()


def test_compile_time_2d_grid_has_no_choice():
    """A 2D grid has no slabs, and 64 x 64 runs on compile-time kernels only,
    so there is nothing to time."""
    from kwave import _lib
    from helpers import case_2d_p0

    inp, record, start, _ = case_2d_p0(n=(64, 64))
    _lib.wisdom_forget()
    r = _lib.tune(inp, record)
    assert r["candidates"] == 0
    assert r["slab_planes"] == 1 and r["streams"] == 1


@pytest.mark.parametrize("radix", [1, 2])
def test_radix_orders_agree_with_the_oracle(tmp_path, radix):
    """Another radix order of the runtime-plan engine (x = 70 = 2 5 7,
    y = 56 = 8 7, z = 48 = 16 3) rounds differently but stays within the
    FP32 parity bar against the oracle, and within 1e-5 of the default order."""
    from kwave import _lib
    from helpers import compare, oracle_outputs

    inp, record, start, _ = case_3d_het(n=(70, 56, 48), nt=24, record=RECORD)
    _lib.wisdom_forget()
    base = _lib.solve(inp, RECORD, start_index=start)
    _forced(tmp_path, inp, radix_plan=radix)
    assert _schedule_of(inp)["radix_plan"] == radix
    other = _lib.solve(inp, RECORD, start_index=start)
    _lib.wisdom_forget()
    errs = compare(other, base)
    assert errs and max(errs.values()) <= 1e-5, errs
    ora = oracle_outputs(inp, RECORD, start, dtype=np.float64)
    errs = compare(other, ora)
    bad = {k: v for k, v in errs.items() if not v <= 1e-4}
    assert not bad, bad
