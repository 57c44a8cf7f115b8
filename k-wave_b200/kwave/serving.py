"""Many independent simulations on one GPU: batched runs and a request server.

The reference runs one simulation per process (``kspaceFirstOrder3DC.m``
starts the binary once per call), so a GPU holding a small grid sits mostly
idle.  Here every simulation is a resident session (``kw_session_*``): its
fields stay in HBM, its time steps are replayed CUDA graphs on its own
stream, and a host scheduler interleaves the sessions' steps in chunks, so
kernels of different simulations overlap on the device.  Simulations never
share device memory, so each result is the same as the same simulation run
alone.

* :func:`run_batch` advances a fixed set of simulations together;
* :class:`Server` admits requests as they arrive, while their estimated
  device memory fits a budget (continuous batching: a request waiting for
  memory is admitted as soon as a finished one frees enough), and records
  each request's time to solution.

Several GPUs: both take a list of devices.  Simulations are independent, so
they are placed whole on one device each, with no collective between
devices: the server puts each request on the device with the most free
budget (the reference's per-run device choice, ``-g`` in
kspaceFirstOrder3DC.m:308-325, made by the scheduler), and the batch runner
deals its simulations out largest first to the least loaded device.

Both take a ``factory`` that builds a session from a request (inputs,
record, start index, device), so the scheduling logic can be exercised
without a GPU.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field

# More hardware work queues than the default 8, so the streams of many
# sessions do not serialise behind one another.  Takes effect only if set
# before the process creates its CUDA context.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


def session_bytes(inp, record, sizes):
    """Device memory a session holds: fields, spectra and medium maps (the
    library's estimate) plus the recorded outputs."""
    dim = 2 if int(inp["Nz"]) == 1 else 3
    ns, nr, ng = int(sizes.num_sensor_points), int(sizes.num_recorded_steps), int(sizes.grid_points)
    per_series = 4 * ns * nr
    b = int(sizes.device_bytes)
    rec = set(record)
    b += per_series * (("p" in rec) + dim * ("u" in rec) + dim * ("u_non_staggered" in rec))
    # rms: the Kahan pair of the completed blocks and the open block's partial sum
    b += 12 * ns * (("p_rms" in rec) + dim * ("u_rms" in rec)) + 4 * ns * 4
    b += 4 * ng * sum(k in rec for k in ("p_max_all", "p_min_all", "p_final"))
    b += 4 * ng * dim * sum(k in rec for k in ("u_max_all", "u_min_all", "u_final"))
    return b


def gpu_session(inp, record, start_index=1, device=-1):
    from ._lib import Session

    return Session(inp, record, start_index, device)


BINARY = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kspaceFirstOrder-B200")
_FLAGS = {"p": "--p_raw", "u": "--u_raw", "u_non_staggered": "--u_non_staggered_raw"}


class DropInSession:
    """One solve the way the reference's C/G-suffixed wrappers run it
    (kspaceFirstOrder3DC.m:159-212, 462-545, 569-776): the input file
    written, the solver binary started, the output file read.  The session
    interface of :func:`gpu_session`, so the plain one-solve-at-a-time
    drop-in can be timed with the same schedulers: ``advance`` runs the
    whole solve."""

    def __init__(self, inp, record, start_index=1, device=-1, workdir=None):
        import tempfile

        self.inp, self.record, self.start, self.device = inp, tuple(record), int(start_index), device
        self.dir = tempfile.mkdtemp(prefix="kwb_dropin_", dir=workdir)
        self.result = None

    def advance(self, n):
        import subprocess

        from . import h5io

        fin, fout = os.path.join(self.dir, "input.h5"), os.path.join(self.dir, "output.h5")
        h5io.write_input_file(fin, self.inp)
        cmd = [BINARY, "-i", fin, "-o", fout, "-s", str(self.start)]
        cmd += [_FLAGS.get(r, "--" + r) for r in self.record]
        if self.device >= 0:
            cmd += ["-g", str(self.device)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"drop-in binary failed ({r.returncode}): {r.stderr.strip()}")
        self.result = h5io.read_output_file(fout, 2 if int(self.inp["Nz"]) == 1 else 3)

    def sync(self):
        pass

    def read(self):
        return self.result

    def close(self):
        import shutil

        shutil.rmtree(self.dir, ignore_errors=True)


def dropin_session(inp, record, start_index=1, device=-1):
    return DropInSession(inp, record, start_index, device)


@dataclass
class Request:
    """One simulation request: the input datasets, what to record, and when
    it arrives (seconds after the server starts)."""
    inp: dict
    record: tuple = ("p",)
    arrival: float = 0.0
    start_index: int = 1
    tag: object = None
    # filled in by the server
    admitted: float = None
    finished: float = None
    result: dict = None
    error: str = None
    nbytes: int = 0
    device: int = None

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival

    @property
    def grid_point_steps(self):
        return int(self.inp["Nx"]) * int(self.inp["Ny"]) * int(self.inp["Nz"]) * int(self.inp["Nt"])


def place_on_devices(inputs, devices):
    """Device of each simulation: largest first (grid-point-steps) to the
    device with the least work so far, so the devices finish together."""
    load = [0] * len(devices)
    out = [None] * len(inputs)
    work = lambda inp: int(inp["Nx"]) * int(inp["Ny"]) * int(inp["Nz"]) * int(inp["Nt"])
    for i in sorted(range(len(inputs)), key=lambda i: -work(inputs[i])):
        k = min(range(len(devices)), key=lambda k: (load[k], k))
        load[k] += work(inputs[i])
        out[i] = devices[k]
    return out


def run_batch(inputs, record=("p",), chunk=25, factory=gpu_session, sync=True, mode="auto", devices=(-1,)):
    """Advance every simulation in `inputs` to its last step and return their
    outputs in order.

    mode "graph": one kw_batch per device advances its simulations, each
    time step of all of them one CUDA graph launch (library sessions only;
    measured a little faster than streams on 48 uneven 3D grids).  mode
    "streams": the sessions are interleaved in chunks of `chunk` steps, each
    session's steps on its own stream, so the device runs them concurrently.
    "auto" takes "graph" for library sessions and "streams" for any other
    session type.  `devices`: the GPUs to spread the simulations over
    (place_on_devices); -1 is the current device.  Work is only enqueued
    until the outputs are read."""
    where = place_on_devices(inputs, list(devices))
    sessions = [factory(inp, record, 1, dev) for inp, dev in zip(inputs, where)]
    try:
        if mode == "auto":
            try:
                from ._lib import Session

                library = all(isinstance(s, Session) for s in sessions)
            except ImportError:
                library = False
            mode = "graph" if library else "streams"
        if mode == "graph":
            from ._lib import Batch

            groups = {}
            for s, dev in zip(sessions, where):
                groups.setdefault(dev, []).append(s)
            batches = [Batch(g) for g in groups.values()]
            try:
                for _ in range(0, max(int(inp["Nt"]) for inp in inputs), chunk):
                    for b in batches:  # each device's batch runs while the host feeds the next
                        b.advance(chunk)
            finally:
                for b in batches:
                    b.close()
        elif mode == "streams":
            left = [int(inp["Nt"]) for inp in inputs]
            while any(left):
                for i, s in enumerate(sessions):
                    if left[i]:
                        n = min(chunk, left[i])
                        s.advance(n)
                        left[i] -= n
        else:
            raise ValueError(f"unknown batch mode {mode!r}")
        return [s.read() for s in sessions] if sync else sessions
    finally:
        if sync:
            for s in sessions:
                s.close()


def run_plain(inputs, record=("p",), factory=gpu_session):
    """The one-simulation-at-a-time drop-in: each simulation runs to its end
    before the next starts."""
    out = []
    for inp in inputs:
        s = factory(inp, record, 1, -1)
        try:
            s.advance(int(inp["Nt"]))
            out.append(s.read())
        finally:
            s.close()
    return out


def library_sizer(r):
    """Device bytes of a request, from the library's output-size query."""
    from ._lib import make_input, make_options, output_sizes

    s, keep = make_input(r.inp)
    return session_bytes(r.inp, r.record, output_sizes(s, make_options(r.record, r.start_index)))


@dataclass
class Server:
    """Admits requests by device-memory budget and interleaves their steps.

    `budget_bytes` bounds the summed estimate of the sessions admitted to
    each device in `devices` (device ordinals, -1 for the current device);
    a request goes to the device with the most free budget.  Each
    session is fed chunks of steps (`chunk`, or if 0 about `chunk_seconds`
    of device time at `step_rate` grid-point-steps/s) while fewer than
    `max_queued` of its chunks are still running, so its stream never runs
    dry while the host is busy elsewhere.  With `priorities`, smaller jobs
    (fewer grid-point-steps) get higher CUDA stream priorities: their
    kernels are scheduled first and the larger jobs' kernels fill the SMs
    they leave idle, so short requests are not held up behind long ones.
    `clock` / `sleep` are the time source (replaceable by a simulated clock
    in tests)."""
    budget_bytes: int = 150 * 10**9
    devices: tuple = (-1,)
    chunk: int = 0
    max_queued: int = 3
    chunk_seconds: float = 4e-3
    step_rate: float = 1e10
    priorities: bool = True
    factory: object = gpu_session
    sizer: object = library_sizer
    clock: object = time.perf_counter
    sleep: object = time.sleep
    idle_sleep_s: float = 2e-4
    log: list = field(default_factory=list)

    def serve(self, requests):
        """Run `requests` to completion in arrival order; returns them with
        admitted / finished times (seconds after start) and results."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            r.nbytes = int(self.sizer(r))
            if r.nbytes > self.budget_bytes:
                r.error = f"needs {r.nbytes} B of device memory, more than the {self.budget_bytes} B budget"
        queue = [r for r in pending if r.error is None]
        levels = self._priority_levels() if self.priorities else None
        active = []  # [request, session, steps queued, chunk, device slot]
        used = [0] * len(self.devices)
        t0 = self.clock()
        now = lambda: self.clock() - t0
        while queue or active:
            progressed = False
            # admission: arrived requests, first come first served, each on
            # the device with the most free budget, while one has room
            while queue and queue[0].arrival <= now():
                k = self.place(queue[0].nbytes, used)
                if k is None:
                    break
                r = queue.pop(0)
                try:
                    sess = self.factory(r.inp, r.record, r.start_index, self.devices[k])
                except Exception as e:  # noqa: BLE001 - reported per request
                    r.error = str(e)
                    continue
                if levels and hasattr(sess, "set_priority"):
                    sess.set_priority(self._priority(r, levels))
                r.admitted = now()
                r.device = self.devices[k]
                used[k] += r.nbytes
                active.append([r, sess, 0, self._chunk(r), k])
                self.log.append(("admit", r.tag, r.admitted, used[k], self.devices[k]))
                progressed = True
            # interleave: top up each session's stream with its next chunk,
            # collect the sessions whose last step has finished
            for a in list(active):
                r, sess, queued, chunk, k = a
                nt = int(r.inp["Nt"])
                if queued < nt:
                    if sess.in_flight() < self.max_queued:
                        n = min(chunk, nt - queued)
                        sess.advance(n)
                        a[2] = queued + n
                        self.log.append(("advance", r.tag, now(), n))
                        progressed = True
                elif sess.in_flight() == 0:
                    try:
                        r.result = sess.read()
                    except Exception as e:  # noqa: BLE001
                        r.error = str(e)
                    finally:
                        sess.close()
                    r.finished = now()
                    used[k] -= r.nbytes
                    active.remove(a)
                    self.log.append(("finish", r.tag, r.finished, used[k], self.devices[k]))
                    progressed = True
            if not progressed:
                self.sleep(self.idle_sleep_s)
        return pending

    def place(self, nbytes, used):
        """Slot of the device with the most free budget that fits `nbytes`
        (the lowest slot on ties), or None when none has room."""
        best = None
        for k, u in enumerate(used):
            if u + nbytes <= self.budget_bytes and (best is None or u < used[best]):
                best = k
        return best

    def _chunk(self, r):
        if self.chunk:
            return self.chunk
        npts = int(r.inp["Nx"]) * int(r.inp["Ny"]) * int(r.inp["Nz"])
        return int(max(5, min(200, self.chunk_seconds * self.step_rate / max(npts, 1))))

    @staticmethod
    def _priority_levels():
        try:
            from ._lib import stream_priority_range

            least, greatest = stream_priority_range()
        except Exception:  # noqa: BLE001 - no device: no priorities
            return None
        return list(range(greatest, least + 1))  # highest priority first

    @staticmethod
    def _priority(r, levels):
        """One level per decade of grid-point-steps above 1e8."""
        import math

        k = int(math.log10(max(r.grid_point_steps, 1))) - 8
        return levels[max(0, min(len(levels) - 1, k))]


def serve_plain(requests, factory=gpu_session, clock=time.perf_counter, sleep=time.sleep):
    """First come, first served, one simulation at a time (the plain drop-in
    behind a queue): the baseline for the server's latencies."""
    pending = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    for r in pending:
        while clock() - t0 < r.arrival:
            sleep(min(1e-3, r.arrival - (clock() - t0)))
        r.admitted = clock() - t0
        sess = factory(r.inp, r.record, r.start_index, -1)
        try:
            sess.advance(int(r.inp["Nt"]))
            r.result = sess.read()
        finally:
            sess.close()
        r.finished = clock() - t0
    return pending


def percentile(values, q):
    v = sorted(values)
    if not v:
        return None
    k = (len(v) - 1) * q / 100.0
    lo, hi = int(k), min(int(k) + 1, len(v) - 1)
    return v[lo] + (v[hi] - v[lo]) * (k - lo)


def summary(requests, elapsed_s=None):
    done = [r for r in requests if r.finished is not None and r.error is None]
    lat = [r.latency for r in done]
    span = elapsed_s if elapsed_s is not None else (max(r.finished for r in done) if done else 0.0)
    gps = sum(r.grid_point_steps for r in done)
    return {"requests": len(requests), "completed": len(done), "failed": sum(r.error is not None for r in requests),
            "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99), "mean_s": sum(lat) / len(lat) if lat else None,
            "makespan_s": span, "grid_pt_steps_per_s": gps / span if span else None}
