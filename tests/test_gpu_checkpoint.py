"""Checkpoints (the external binaries' --checkpoint_file): a run saved
between two steps and resumed in a fresh session finishes bit for bit like
the uninterrupted run, through the session API and through the file run."""
import os

import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert set(a) == set(b)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("stop", [1, 17])
def test_session_resume_is_bit_exact_2d_initial_pressure(tmp_path, stop):
    from kwave import _lib

    inp, record, start, _ = case_2d_p0(n=(64, 48), nt=40, record=("p", "p_max", "p_rms", "u", "p_final"))
    want = _lib.solve(inp, record, start_index=3)
    s = _lib.Session(inp, record, start_index=3)
    s.advance(stop)
    s.save(tmp_path / "c.h5")
    s.close()
    r = _lib.Session(inp, record, start_index=3)
    r.restore(tmp_path / "c.h5")
    assert r.steps_done == stop
    r.advance(40 - stop)
    _same(r.read(), want)
    r.close()


def test_session_resume_is_bit_exact_3d_source_absorbing(tmp_path):
    from kwave import _lib

    rec = ("p", "p_rms", "u_max", "u_non_staggered", "p_max_all")
    inp, _, start, _ = case_3d_het(n=(36, 30, 32), nt=45, record=rec)
    want = _lib.solve(inp, rec)
    s = _lib.Session(inp, rec)
    s.advance(20)  # the tone burst is still on: sources resume mid-signal
    s.save(tmp_path / "c.h5")
    s.close()
    r = _lib.Session(inp, rec)
    r.restore(tmp_path / "c.h5")
    r.advance(25)
    _same(r.read(), want)
    r.close()


def test_file_run_with_checkpoints_and_resume(tmp_path):
    from kwave import _lib, h5io

    rec = ("p", "p_max")
    inp, _, _, _ = case_3d_het(n=(32, 32, 32), nt=40, record=rec, seed=11)
    fin, fout, ck = tmp_path / "in.h5", tmp_path / "out.h5", tmp_path / "ck.h5"
    h5io.write_input_file(fin, inp)
    _lib.run_file(fin, fout, rec, checkpoint=ck, checkpoint_timesteps=7)
    assert not ck.exists()  # removed once the output is written
    plain = h5io.read_output_file(fout, 3)
    _same(plain, _lib.solve(inp, rec))
    # an interrupted run: state after 23 steps on disk, then the file run resumes it
    s = _lib.Session(inp, rec)
    s.advance(23)
    s.save(ck)
    s.close()
    os.remove(fout)
    _lib.run_file(fin, fout, rec, checkpoint=ck, checkpoint_timesteps=10)
    _same(h5io.read_output_file(fout, 3), plain)


def test_restore_rejects_what_it_cannot_continue(tmp_path):
    from kwave import _lib, h5io

    inp, record, start, _ = case_2d_p0(n=(64, 48), nt=20, record=("p",))
    s = _lib.Session(inp, ("p",))
    s.advance(5)
    s.save(tmp_path / "c.h5")
    with pytest.raises(_lib.KwaveError) as e:
        s.restore(tmp_path / "c.h5")  # not a fresh session
    assert e.value.code == _lib.KW_ERR_INVALID_ARGUMENT
    s.close()
    other, _, _, _ = case_2d_p0(n=(60, 48), nt=20, record=("p",))
    r = _lib.Session(other, ("p",))
    with pytest.raises(_lib.KwaveError) as e:
        r.restore(tmp_path / "c.h5")
    assert e.value.code == _lib.KW_ERR_INVALID_ARGUMENT and "different" in str(e.value)
    r.close()
    r = _lib.Session(inp, ("p", "p_max"))
    with pytest.raises(_lib.KwaveError) as e:
        r.restore(tmp_path / "c.h5")  # p_max was not recorded in the checkpointed run
    assert "p_max" in str(e.value)
    r.close()
    h5io.write_input_file(tmp_path / "in.h5", inp)
    r = _lib.Session(inp, ("p",))
    with pytest.raises(_lib.KwaveError) as e:
        r.restore(tmp_path / "in.h5")
    assert e.value.code == _lib.KW_ERR_IO
    r.close()
