"""Batched and served simulations on the GPU: every result is bit for bit the
result of the same simulation solved alone (sessions share no device
memory and the kernels are deterministic), whatever runs beside it."""
import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het

pytestmark = pytest.mark.gpu


def _cases():
    return [
        (case_2d_p0(n=(64, 48), nt=60)[0], ("p", "p_max", "u")),
        (case_3d_het(n=(36, 30, 32), nt=45, record=("p", "p_rms"))[0], ("p", "p_rms")),
        (case_2d_p0(n=(75, 60), nt=33)[0], ("p", "p_final")),
        (case_3d_het(n=(32, 32, 32), nt=52, absorbing=False, record=("p", "p_max"), seed=3)[0], ("p", "p_max")),
    ]


def _same(a, b):
    assert set(a) == set(b)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_batch_results_equal_solo_results():
    from kwave import _lib, serving

    cases = _cases()
    alone = [_lib.solve(inp, rec) for inp, rec in cases]
    # one record list per batch: run each case's record set as its own batch member
    sessions = [serving.gpu_session(inp, rec) for inp, rec in cases]
    try:
        left = [int(inp["Nt"]) for inp, _ in cases]
        while any(left):
            for i, s in enumerate(sessions):
                if left[i]:
                    n = min(7, left[i])
                    s.advance(n)
                    left[i] -= n
        mixed = [s.read() for s in sessions]
    finally:
        for s in sessions:
            s.close()
    for a, m in zip(alone, mixed):
        _same(a, m)


def test_run_batch_matches_plain():
    from kwave import serving

    inputs = [case_2d_p0(n=(48, 48), nt=40)[0], case_2d_p0(n=(60, 50), nt=25)[0], case_2d_p0(n=(32, 64), nt=31)[0]]
    a = serving.run_batch(inputs, ("p", "p_max"), chunk=9)
    b = serving.run_plain(inputs, ("p", "p_max"))
    for x, y in zip(a, b):
        _same(x, y)


def test_server_results_equal_solo_results_under_a_budget():
    from kwave import _lib, serving

    cases = _cases()
    reqs = [serving.Request(inp=inp, record=rec, arrival=0.02 * i, tag=i) for i, (inp, rec) in enumerate(cases)]
    sizes = [serving.library_sizer(r) for r in reqs]
    budget = sorted(sizes)[-1] + sorted(sizes)[-2]  # room for about two at a time
    srv = serving.Server(budget_bytes=budget, chunk=8)
    out = srv.serve(reqs)
    for r, (inp, rec) in zip(sorted(out, key=lambda r: r.tag), cases):
        assert r.error is None, r.error
        _same(r.result, _lib.solve(inp, rec))
        assert r.admitted >= r.arrival and r.finished > r.admitted
    assert max(e[3] for e in srv.log if e[0] == "admit") <= budget
    stats = serving.summary(out)
    assert stats["completed"] == len(cases) and stats["p99_s"] >= stats["p50_s"] > 0


def test_in_flight_reports_running_chunks():
    from kwave import _lib

    inp = case_3d_het(n=(64, 64, 64), nt=200, record=("p",))[0]
    s = _lib.Session(inp, ("p",))
    try:
        s.advance(100)
        s.advance(100)
        assert s.in_flight() in (0, 1, 2)
        s.sync()
        assert s.in_flight() == 0
    finally:
        s.close()


def test_dropin_sessions_give_the_same_results():
    """The plain drop-in baseline (solver binary per request, files in and
    out) returns what the resident sessions return, bit for bit."""
    from kwave import serving

    cases = _cases()[:3]
    reqs = [serving.Request(inp=inp, record=rec, arrival=0.0, tag=i) for i, (inp, rec) in enumerate(cases)]
    dropped = serving.serve_plain(reqs, factory=serving.dropin_session)
    for r, (inp, rec) in zip(dropped, cases):
        s = serving.gpu_session(inp, rec)
        s.advance(int(inp["Nt"]))
        _same(r.result, s.read())
        s.close()


def test_server_over_two_device_slots_gives_solo_results():
    """Placement across devices, with both slots naming device 0 (this run
    has one GPU): requests are spread over the two budgets and each result is
    still the solo result."""
    from kwave import _lib, serving

    cases = _cases()
    reqs = [serving.Request(inp=inp, record=rec, arrival=0.0, tag=i) for i, (inp, rec) in enumerate(cases)]
    sizes = [serving.library_sizer(r) for r in reqs]
    srv = serving.Server(budget_bytes=max(sizes) + min(sizes), chunk=8, devices=(0, 0))
    out = srv.serve(reqs)
    slots = [e for e in srv.log if e[0] == "admit"]
    assert len(slots) == len(cases)
    for r, (inp, rec) in zip(sorted(out, key=lambda r: r.tag), cases):
        assert r.error is None, r.error
        assert r.device == 0
        _same(r.result, _lib.solve(inp, rec))


def test_run_batch_over_two_device_slots_matches_plain():
    from kwave import serving

    inputs = [case_2d_p0(n=(48, 48), nt=40)[0], case_2d_p0(n=(60, 50), nt=25)[0], case_2d_p0(n=(32, 64), nt=31)[0]]
    a = serving.run_batch(inputs, ("p", "p_max"), chunk=9, devices=(0, 0))
    b = serving.run_plain(inputs, ("p", "p_max"))
    for x, y in zip(a, b):
        _same(x, y)
