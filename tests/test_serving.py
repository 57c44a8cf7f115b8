"""The batch runner and request server's scheduling, without a GPU: fake
sessions whose chunks take simulated time on a simulated clock."""
import numpy as np
import pytest

from kwave import serving


class Clock:
    def __init__(self):
        self.t = 0.0

    def now(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeSession:
    """Each chunk of n steps occupies the session's stream for n * cost
    simulated seconds; sessions run side by side."""

    def __init__(self, clock, inp, record, start_index=1, cost=1e-3, trace=None):
        self.clock, self.inp, self.cost = clock, inp, cost
        self.ends = []
        self.steps = 0
        self.closed = False
        self.trace = trace if trace is not None else []

    def advance(self, n):
        start = max([self.clock.now()] + self.ends[-1:])
        self.ends.append(start + n * self.cost)
        self.steps += n
        self.trace.append((self.inp["tag"], n))

    def in_flight(self):
        return sum(e > self.clock.now() for e in self.ends)

    def read(self):
        assert self.steps == self.inp["Nt"] and self.in_flight() == 0
        return {"p": np.full(3, float(self.inp["tag"]))}

    def close(self):
        self.closed = True


def _req(tag, nt=100, arrival=0.0, nbytes=1):
    return serving.Request(inp={"Nx": 4, "Ny": 4, "Nz": 1, "Nt": nt, "tag": tag, "bytes": nbytes}, arrival=arrival,
                           tag=tag)


def _server(clock, budget, trace=None, chunk=10, devices=(-1,)):
    made = []

    def factory(inp, record, start_index=1, device=-1):
        s = FakeSession(clock, inp, record, start_index, trace=trace)
        s.device = device
        made.append(s)
        return s

    srv = serving.Server(budget_bytes=budget, chunk=chunk, factory=factory, sizer=lambda r: r.inp["bytes"],
                         priorities=False, clock=clock.now, sleep=clock.sleep, idle_sleep_s=1e-4, devices=devices)
    return srv, made


def test_budget_bounds_the_admitted_sessions_and_order_is_fifo():
    clock = Clock()
    srv, made = _server(clock, budget=2)
    reqs = [_req(i) for i in range(5)]
    out = srv.serve(reqs)
    assert all(r.error is None and r.result is not None for r in out)
    assert all(int(r.result["p"][0]) == r.tag for r in out)
    assert all(s.closed for s in made)
    admits = [e for e in srv.log if e[0] == "admit"]
    assert [e[1] for e in admits] == [0, 1, 2, 3, 4]
    assert max(e[3] for e in admits) <= 2
    # with room for two, the third waits for the first to finish
    fin = {e[1]: e[2] for e in srv.log if e[0] == "finish"}
    assert dict((e[1], e[2]) for e in admits)[2] >= min(fin[0], fin[1])


def test_oversized_request_is_rejected_and_the_rest_complete():
    clock = Clock()
    srv, _ = _server(clock, budget=3)
    reqs = [_req(0), _req(1, nbytes=4), _req(2)]
    out = srv.serve(reqs)
    assert out[1].error and "budget" in out[1].error and out[1].result is None
    assert out[0].result is not None and out[2].result is not None


def test_steps_of_active_sessions_interleave():
    clock = Clock()
    trace = []
    srv, _ = _server(clock, budget=10, trace=trace)
    srv.serve([_req(0, nt=100), _req(1, nt=100)])
    first = [t for t, _ in trace[:6]]
    assert set(first) == {0, 1}  # both progress before either finishes
    # a session never has more than max_queued chunks running
    assert sum(n for t, n in trace if t == 0) == 100


def test_late_request_is_admitted_while_a_long_one_runs():
    clock = Clock()
    srv, _ = _server(clock, budget=10)
    reqs = [_req(0, nt=2000), _req(1, nt=50, arrival=0.05)]
    out = srv.serve(reqs)
    long, short = out
    assert short.admitted >= 0.05 and short.admitted < long.finished
    assert short.finished < long.finished
    assert short.latency < 0.5 * long.latency


def test_admission_waits_for_arrival_times():
    clock = Clock()
    srv, _ = _server(clock, budget=10)
    reqs = [_req(i, nt=10, arrival=0.1 * i) for i in range(4)]
    out = srv.serve(reqs)
    for r in out:
        assert r.admitted >= r.arrival - 1e-12
        assert r.finished > r.admitted


def test_batch_and_plain_return_outputs_in_order():
    clock = Clock()
    mk = lambda inp, record, start_index=1, device=-1: FakeSession(clock, inp, record, cost=0.0)
    inputs = [{"Nx": 4, "Ny": 4, "Nz": 1, "Nt": nt, "tag": i} for i, nt in enumerate((30, 7, 55))]
    a = serving.run_batch(inputs, ("p",), chunk=10, factory=mk)
    b = serving.run_plain(inputs, ("p",), factory=mk)
    assert [int(x["p"][0]) for x in a] == [0, 1, 2] == [int(x["p"][0]) for x in b]


def test_summary_percentiles():
    reqs = [_req(i) for i in range(5)]
    for i, r in enumerate(reqs):
        r.finished = 1.0 + i
    s = serving.summary(reqs)
    assert s["completed"] == 5 and s["p50_s"] == pytest.approx(3.0) and s["p99_s"] == pytest.approx(4.96)
    assert serving.percentile([], 50) is None


def test_session_bytes_counts_recorded_outputs():
    class Sz:
        num_sensor_points, num_recorded_steps, grid_points, device_bytes = 10, 100, 1000, 5000

    inp = {"Nz": 1}
    base = serving.session_bytes(inp, ("p_max",), Sz)
    assert serving.session_bytes(inp, ("p",), Sz) - serving.session_bytes(inp, (), Sz) == 4 * 10 * 100
    assert serving.session_bytes(inp, ("u",), Sz) - serving.session_bytes(inp, (), Sz) == 2 * 4 * 10 * 100
    assert serving.session_bytes(inp, ("p_final",), Sz) - serving.session_bytes(inp, (), Sz) == 4 * 1000
    # rms: a Kahan pair of the completed blocks and the open block's partial sum per sensor point
    assert serving.session_bytes(inp, ("p_rms",), Sz) - serving.session_bytes(inp, (), Sz) == 12 * 10
    assert serving.session_bytes(inp, ("u_rms",), Sz) - serving.session_bytes(inp, (), Sz) == 2 * 12 * 10
    assert base >= 5000


def test_priority_levels_follow_job_size_and_chunks_follow_grid_size():
    levels = [-5, -4, -3, -2, -1, 0]
    small = serving.Request(inp={"Nx": 256, "Ny": 256, "Nz": 1, "Nt": 500})        # 3.3e7 steps
    mid = serving.Request(inp={"Nx": 128, "Ny": 128, "Nz": 128, "Nt": 800})        # 1.7e9
    big = serving.Request(inp={"Nx": 256, "Ny": 256, "Nz": 256, "Nt": 1500})       # 2.5e10
    p = [serving.Server._priority(r, levels) for r in (small, mid, big)]
    assert p == [-5, -4, -3] and p == sorted(p)
    srv = serving.Server(chunk=0, chunk_seconds=4e-3, step_rate=1e10)
    assert srv._chunk(small) == 200 and srv._chunk(big) == 5
    assert serving.Server(chunk=17)._chunk(big) == 17


def test_requests_go_to_the_device_with_the_most_free_budget():
    clock = Clock()
    srv, made = _server(clock, budget=4, devices=(0, 1))
    reqs = [_req(0, nbytes=3), _req(1, nbytes=2), _req(2, nbytes=2), _req(3, nbytes=1)]
    out = srv.serve(reqs)
    assert all(r.error is None and int(r.result["p"][0]) == r.tag for r in out)
    # 0 -> device 0 (both empty, lowest first); 1 -> device 1 (4 free against 1);
    # 2 -> device 1 (2 free against 1); 3 -> device 0 (1 free against 0)
    assert [r.device for r in out] == [0, 1, 1, 0]
    assert [s.device for s in made] == [0, 1, 1, 0]
    for dev in (0, 1):  # no device ever holds more than its budget
        assert max(e[3] for e in srv.log if e[0] == "admit" and e[4] == dev) <= 4


def test_a_request_waits_until_some_device_has_room():
    clock = Clock()
    srv, _ = _server(clock, budget=3, devices=(0, 1))
    reqs = [_req(0, nbytes=3, nt=200), _req(1, nbytes=3, nt=100), _req(2, nbytes=3, nt=10)]
    out = srv.serve(reqs)
    assert [r.device for r in out[:2]] == [0, 1]
    # the third fits nowhere until the shorter of the first two finishes, and takes its device
    assert out[2].admitted >= out[1].finished and out[2].device == 1


def test_two_devices_halve_the_makespan_of_equal_jobs():
    def makespan(devices):
        clock = Clock()
        srv, _ = _server(clock, budget=1, devices=devices)
        out = srv.serve([_req(i, nt=100) for i in range(4)])
        return max(r.finished for r in out)

    one, two = makespan((0,)), makespan((0, 1))
    assert two == pytest.approx(one / 2, rel=0.05)


def test_batch_placement_balances_work_largest_first():
    inputs = [{"Nx": n, "Ny": n, "Nz": n, "Nt": 10} for n in (64, 128, 96, 128, 64)]
    where = serving.place_on_devices(inputs, [0, 1])
    work = lambda i: inputs[i]["Nx"] ** 3
    load = {d: sum(work(i) for i in range(5) if where[i] == d) for d in (0, 1)}
    # the two 128^3 jobs land on different devices, the rest fill the lighter one
    assert where[1] != where[3]
    assert abs(load[0] - load[1]) <= 96 ** 3
    clock = Clock()
    made = []

    def mk(inp, record, start_index=1, device=-1):
        s = FakeSession(clock, dict(inp, tag=len(made)), record, cost=0.0)
        s.device = device
        made.append(s)
        return s

    serving.run_batch([dict(i) for i in inputs], ("p",), chunk=5, factory=mk, devices=(0, 1))
    assert [s.device for s in made] == where
