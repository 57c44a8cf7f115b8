"""Wisdom files of the launch-schedule tuner, read and written without a GPU
(kw_wisdom_import / kw_wisdom_export / kw_wisdom_forget)."""
import pytest

from kwave import _lib


def _entries(path):
    return sorted(l.split() for l in open(path) if l.strip() and not l.startswith("#"))


def test_import_export_round_trip_and_merge(tmp_path):
    a = tmp_path / "a.txt"
    a.write_text("# comment\n256x256x256/eos1/nl1/as0/dense1/sm10.0148 128 2 8 16 0 1.299\n"
                 "100x120x90/eos1/nl0/as0/dense0/sm10.0148 90 1 4 8 2 0.48\n")
    _lib.wisdom_forget()
    _lib.wisdom_import(str(a))
    out = tmp_path / "out.txt"
    out.write_text("64x48x40/eos1/nl1/as0/dense0/sm10.0148 20 2 8 16 1 0.05\n")
    _lib.wisdom_export(str(out))  # merges: the file's entry stays, the table's are added
    got = _entries(out)
    assert [e[0] for e in got] == sorted(["256x256x256/eos1/nl1/as0/dense1/sm10.0148",
                                          "100x120x90/eos1/nl0/as0/dense0/sm10.0148",
                                          "64x48x40/eos1/nl1/as0/dense0/sm10.0148"])
    row = dict((e[0], e[1:]) for e in got)["256x256x256/eos1/nl1/as0/dense1/sm10.0148"]
    assert row[:5] == ["128", "2", "8", "16", "0"] and abs(float(row[5]) - 1.299) < 1e-6
    assert dict((e[0], e[1:]) for e in got)["100x120x90/eos1/nl0/as0/dense0/sm10.0148"][4] == "2"
    _lib.wisdom_forget()
    empty = tmp_path / "empty.txt"
    _lib.wisdom_export(str(empty))
    assert _entries(empty) == []


@pytest.mark.parametrize("text", ["key 1 2 3\n", "key 0 1 8 16 0 1.0\n", "key 4 3 8 16 0 1.0\n",
                                  "key 4 2 8 16 3 1.0\n", "key 4 2 8 16 1.0\n", "key a b c d e f\n"])
def test_malformed_wisdom_is_rejected(tmp_path, text):
    p = tmp_path / "bad.txt"
    p.write_text(text)
    _lib.wisdom_forget()
    with pytest.raises(_lib.KwaveError, match="wisdom"):
        _lib.wisdom_import(str(p))
    with pytest.raises(_lib.KwaveError):
        _lib.wisdom_import(str(tmp_path / "missing.txt"))


def test_tuner_and_batch_entry_points_reject_bad_arguments():
    """Argument checks of kw_tune / kw_batch_* / kw_session_schedule that run
    before any device work."""
    import ctypes as C

    st = _lib.KwStatus()
    sc = _lib.KwSchedule()
    assert _lib.lib.kw_tune(None, None, C.byref(sc), C.byref(st)) == _lib.KW_ERR_INVALID_ARGUMENT
    h = C.c_void_p()
    assert _lib.lib.kw_batch_create(None, 0, C.byref(h), C.byref(st)) == _lib.KW_ERR_INVALID_ARGUMENT
    arr = (C.c_void_p * 2)(None, None)
    assert _lib.lib.kw_batch_create(arr, 2, C.byref(h), C.byref(st)) == _lib.KW_ERR_INVALID_ARGUMENT
    assert b"NULL session" in st.message
    assert not h.value
    assert _lib.lib.kw_batch_advance(None, 1, C.byref(st)) == _lib.KW_ERR_INVALID_ARGUMENT
    assert _lib.lib.kw_batch_graph_launches(None) == 0
    assert _lib.lib.kw_session_schedule(None, C.byref(sc)) == _lib.KW_ERR_INVALID_ARGUMENT
    _lib.lib.kw_batch_destroy(None)
