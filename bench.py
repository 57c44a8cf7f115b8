"""Benchmark: grid-point-steps/s of the k-space fluid time loop.

Workload: 3D 256^3 (PML 10 inside), heterogeneous (smoothed-noise c and rho),
power-law absorbing (alpha 0.75 dB/(MHz^y cm), y 1.5), nonlinear (B/A 6),
48x48 additive plane pressure source (1 MHz 3-cycle tone burst, 1 MPa),
every grid point a sensor recording p_max and p_rms, Nt 1200, FP32.

A "step" is one time step of that simulation.  `value` is measured with the
simulation resident in HBM (kw_session_advance, CUDA events on the session's
stream); `e2e` is a whole solve through the C ABI (kw_solve) from pinned
host buffers, host<->device copies included.  Every field (1.1 GB working
set) is larger than the 126 MB L2, so no flush is needed between steps.
Before anything is timed, kw_tune picks the step's launch schedule for the
grid (z slabs, streams; reported in `schedule`); the session and the
solves use it.

The `batched` object times 48 uneven 3D simulations one at a time, as
sessions interleaved on their own streams, and as one kw_batch (each step of
all 48 one CUDA graph launch), plus the plain drop-in (the solver binary per
simulation); `served` a Poisson request stream through the server.

Multi-GPU: each rank runs its own independent simulation ("replicas
only": one simulation does not shard), so `value` sums over ranks.

`--impl reference` times the reference algorithm on the host CPU instead:
the reference's own implementation is MATLAB (not installable here), so the
CPU restatement in oracle/ (numpy + scipy.fft on all host threads) stands
in for it.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

# Streams of concurrent simulations (the batched and served samples) need
# more hardware work queues than the default 8; set before CUDA starts.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "k-wave_b200"))
sys.path.insert(0, ROOT)

METRIC = "grid-pt-steps/s at 256^3 FP32 (heterogeneous absorbing nonlinear)"
UNIT = "grid-pt-steps/s"
B_ALG = 232.0  # algorithmic bytes per grid-point-step (58 FP32 full-grid arrays)
WORKLOAD = "3D 256^3 het absorbing nonlinear, additive plane p source, all-point p_max/p_rms, Nt 1200, FP32"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_input(n, nt, shape=None):
    from kwave.simulation import prepare
    from kwave.workloads import het_absorbing_3d

    kg, medium, source, sensor = het_absorbing_3d(n=n, nt=nt, shape=shape)
    inp, record, start, _ = prepare(kg, medium, source, sensor)
    return inp, record, start


def pin_inputs(inp):
    """Copy every array input into pinned host memory, flattened x-fastest."""
    import torch

    out = {}
    npts = int(inp["Nx"]) * int(inp["Ny"]) * int(inp["Nz"])
    for k, v in inp.items():
        if isinstance(v, np.ndarray) and (v.size == npts or k.endswith("index")):
            dt = np.uint64 if k.endswith("index") or k.endswith("corners") else np.float32
            flat = np.asarray(v).reshape(-1, order="F").astype(dt)
            t = torch.empty(flat.size, dtype=torch.float32 if dt == np.float32 else torch.int64, pin_memory=True)
            a = t.numpy()
            if dt == np.uint64:
                a = a.view(np.uint64)
            a[...] = flat
            out[k] = a
            out["_pin_" + k] = t
        else:
            out[k] = v
    return out


def h2d_bytes(inp):
    b = 0
    for k, v in inp.items():
        if k.startswith("_pin_"):
            continue
        if isinstance(v, np.ndarray):
            b += v.nbytes if v.dtype != np.float64 else v.size * 4
    return b


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def traffic_per_step(n):
    """DRAM bytes per step from the committed ncu summary (scaled to n^3)."""
    path = os.path.join(ROOT, "profiles", "step_het_absorbing_traffic.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_grid_point_step:\s*([0-9.eE+-]+)", txt)
    if not m:
        return None
    return float(m.group(1)) * n ** 3


def cpu_sample(inp, record, steps=5, warmup=2):
    """Time the oracle (numpy/scipy, all host threads) on the first
    warmup+steps time steps of the same workload."""
    from oracle.kspace_oracle import simulate

    stamps = []
    simulate(inp, record=record, dtype=np.float32, workers=-1, max_steps=warmup + steps,
             on_step=lambda t: stamps.append(time.perf_counter()))
    per = (stamps[-1] - stamps[warmup - 1]) / steps
    npts = int(inp["Nx"]) * int(inp["Ny"]) * int(inp["Nz"])
    return npts / per, per, warmup, steps


def replica_throughput(ms_local, units_local, dist=None, device=None):
    """Whole-job throughput of independent replicas: the units all ranks
    processed divided by the slowest rank's time (max over ranks).  Every
    rank calls it (it is a collective when `dist` is given)."""
    import torch

    t = torch.tensor([float(ms_local), float(units_local)], dtype=torch.float64, device=device)
    if dist is not None:
        ms = t[:1].clone()
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        units = t[1:].clone()
        dist.all_reduce(units, op=dist.ReduceOp.SUM)
        t = torch.cat([ms, units])
    ms_max, units_all = float(t[0]), float(t[1])
    return units_all / (ms_max / 1e3), ms_max


def _lib_batch(sessions):
    from kwave import _lib

    return _lib.Batch(sessions)


def batched_sample(n_sims, nt, chunk=25):
    """Config of many independent 3D linear lossy simulations on uneven
    2^a 3^b 5^c grids (64..192 per edge): grid-point-steps/s when they advance
    together (run_batch) and one at a time (the plain drop-in).  Sessions are
    created before either timed region; each region is bracketed by a device
    synchronize and timed on the host clock (work on many streams)."""
    import torch

    from kwave import serving
    from kwave.simulation import prepare
    from kwave.workloads import uneven_lossy_3d

    inputs = []
    for i in range(n_sims):
        kg, medium, source, sensor = uneven_lossy_3d(i, n_sims=n_sims, nt=nt)
        inp, record, start, _ = prepare(kg, medium, source, sensor)
        inputs.append(inp)
    work = sum(int(i["Nx"]) * int(i["Ny"]) * int(i["Nz"]) * int(i["Nt"]) for i in inputs)
    for inp in inputs:  # warm-up outside the timed runs: loads each kernel length, captures a step graph
        s_ = serving.gpu_session(inp, record)
        s_.advance(3)
        s_.sync()
        s_.close()
    res = {}
    # end to end, as a user sees it: the batch including its sessions'
    # set-up, uploads and read-back, against the plain drop-in -- each
    # simulation through the solver binary, input file in, output file out,
    # one at a time (what kspaceFirstOrder3DG with 'BinaryName' does)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    outs = serving.run_batch(inputs, record=tuple(record), chunk=chunk)
    torch.cuda.synchronize()
    res["batched_e2e"] = work / (time.perf_counter() - t0)
    # the drop-in on every third simulation (each run costs a process and a
    # CUDA context, about a second on these machines): its rate is compared
    sample = list(range(0, n_sims, 3))
    t0 = time.perf_counter()
    same = True
    for i in sample:
        s_ = serving.dropin_session(inputs[i], record)
        s_.advance(int(inputs[i]["Nt"]))
        r = s_.read()
        s_.close()
        same = same and all(np.array_equal(r[k], outs[i][k]) for k in outs[i])
    work_s = sum(int(inputs[i]["Nx"]) * int(inputs[i]["Ny"]) * int(inputs[i]["Nz"]) * int(inputs[i]["Nt"])
                 for i in sample)
    res["plain_dropin"] = work_s / (time.perf_counter() - t0)
    for mode in ("plain", "batched", "batched_graph"):
        sessions = [serving.gpu_session(inp, record) for inp in inputs]
        for s_ in sessions:
            s_.sync()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if mode == "plain":
            for s_, inp in zip(sessions, inputs):
                s_.advance(int(inp["Nt"]))
                s_.sync()
        elif mode == "batched_graph":  # one kw_batch: each step of all 48 one graph launch
            b = _lib_batch(sessions)
            for _ in range(0, max(int(i["Nt"]) for i in inputs), chunk):
                b.advance(chunk)
            b.sync()
            res["graph_launches"] = b.graph_launches
            b.close()
        else:
            left = [int(i["Nt"]) for i in inputs]
            while any(left):
                for k, s_ in enumerate(sessions):
                    if left[k]:
                        m = min(chunk, left[k])
                        s_.advance(m)
                        left[k] -= m
            for s_ in sessions:
                s_.sync()
        torch.cuda.synchronize()
        res[mode] = work / (time.perf_counter() - t0)
        if mode == "batched_graph":
            same = same and all(all(np.array_equal(r[k], o[k]) for k in o)
                                for r, o in zip((s_.read() for s_ in sessions), outs))
        for s_ in sessions:
            s_.close()
    return {"workload": f"{n_sims} independent 3D linear lossy sims, edges 64..192 (5-smooth), y 1.1, "
                        f"200 sensor points, Nt {nt}, FP32", "unit": UNIT,
            "batched": res["batched"], "plain": res["plain"], "speedup": res["batched"] / res["plain"],
            "batched_graph": res["batched_graph"], "graph_speedup": res["batched_graph"] / res["plain"],
            "graph_launches": res["graph_launches"],
            "batched_e2e": res["batched_e2e"], "plain_dropin": res["plain_dropin"],
            "speedup_vs_dropin": res["batched_e2e"] / res["plain_dropin"], "results_identical": same,
            "timing": "host clock around a device synchronize.  batched / plain: resident sessions created "
                      "before the timed region, advanced together (each on its own stream) / one at a time.  "
                      "batched_graph: the same sessions in one kw_batch, each time step of all of them one "
                      "CUDA graph launch.  batched_e2e: run_batch "
                      "including set-up, uploads and read-back.  plain_dropin: every third simulation, each "
                      "with its input file written, the solver binary run and the output file read, one at a "
                      "time (grid-point-steps of those simulations / their wall time)"}


def served_sample(n_requests, budget_gb=150.0, chunk=0):
    """Seeded Poisson stream (20 requests/s) of 2D 256^2..1024^2 and 3D
    64^3..256^3 solves, half absorbing, Nt 300..1500: time to solution p50 /
    p99 and aggregate grid-point-steps/s, for the server (admission by
    device-memory budget, interleaved steps) and for first-come-first-served
    one-at-a-time solves."""
    from kwave import serving
    from kwave.simulation import prepare
    from kwave.workloads import served_request

    def requests():
        out = []
        for i in range(n_requests):
            arrival, (kg, medium, source, sensor) = served_request(i)
            inp, record, start, _ = prepare(kg, medium, source, sensor, pml_size=10)
            out.append(serving.Request(inp=inp, record=tuple(record), arrival=arrival, start_index=start, tag=i))
        return out

    reqs = requests()
    for r in reqs:  # warm-up outside the timed runs: loads each kernel length, captures a step graph
        s_ = serving.gpu_session(r.inp, r.record, r.start_index)
        s_.advance(3)
        s_.sync()
        s_.close()
    srv = serving.Server(budget_bytes=int(budget_gb * 1e9), chunk=chunk)
    t0 = time.perf_counter()
    served = srv.serve(reqs)
    s_served = serving.summary(served, time.perf_counter() - t0)
    plain_reqs = [serving.Request(inp=r.inp, record=r.record, arrival=r.arrival, start_index=r.start_index, tag=r.tag)
                  for r in reqs]
    t0 = time.perf_counter()
    plain = serving.serve_plain(plain_reqs)
    s_plain = serving.summary(plain, time.perf_counter() - t0)
    same = all(np.array_equal(a.result[k], b.result[k]) for a, b in zip(served, plain) for k in a.result)
    # the plain drop-in behind the same queue: each request through the solver
    # binary (input file, binary, output file), first come first served
    drop_reqs = [serving.Request(inp=r.inp, record=r.record, arrival=r.arrival, start_index=r.start_index, tag=r.tag)
                 for r in reqs]
    t0 = time.perf_counter()
    dropped = serving.serve_plain(drop_reqs, factory=serving.dropin_session)
    s_drop = serving.summary(dropped, time.perf_counter() - t0)
    same = same and all(np.array_equal(a.result[k], b.result[k]) for a, b in zip(served, dropped) for k in a.result)
    return {"workload": f"{n_requests} requests, Poisson 20/s (seed 5): 2D 256^2..1024^2 / 3D 64^3..256^3, "
                        "half absorbing (y 1.0-1.8), Nt 300..1500, plane tone-burst source, FP32",
            "budget_gb": budget_gb, "served": s_served, "plain": s_plain, "plain_dropin": s_drop,
            "p50_speedup": s_plain["p50_s"] / s_served["p50_s"] if s_served["p50_s"] else None,
            "p99_speedup": s_plain["p99_s"] / s_served["p99_s"] if s_served["p99_s"] else None,
            "throughput_speedup": (s_served["grid_pt_steps_per_s"] / s_plain["grid_pt_steps_per_s"]
                                   if s_plain["grid_pt_steps_per_s"] else None),
            "vs_dropin": {"p50_speedup": s_drop["p50_s"] / s_served["p50_s"] if s_served["p50_s"] else None,
                          "p99_speedup": s_drop["p99_s"] / s_served["p99_s"] if s_served["p99_s"] else None,
                          "throughput_speedup": (s_served["grid_pt_steps_per_s"] / s_drop["grid_pt_steps_per_s"]
                                                 if s_drop["grid_pt_steps_per_s"] else None)},
            "results_identical": same,
            "timing": "host clock from the first arrival; latency = finish - arrival.  plain: in-process "
                      "kw_solve one at a time; plain_dropin: the solver binary per request (input file "
                      "written, binary run, output file read), one at a time"}


def workload_config(grid, nt, world):
    """The `config` object of both arms (same keys, same values)."""
    return {"workload": WORKLOAD, "grid": [int(g) for g in grid], "Nt": int(nt),
            "parallelism": f"replicas{world}", "l2": "working set 1.1 GB > 126 MB L2, no flush needed"}


def mapped_repo_libraries():
    """Shared objects of this repository mapped into the process."""
    try:
        with open("/proc/self/maps") as f:
            return sorted({ln.split()[-1] for ln in f if ln.rstrip().endswith(".so") and ROOT in ln})
    except OSError:
        return []


class _SampleDone(Exception):
    pass


def fft_sample(grids=((256, 256, 256), (120, 150, 90), (160, 135, 192)), reps=20, warmup=3):
    """The solver's own FFT passes (kw_fft3d: x row transform, y and z column
    passes) against cuFFT (torch.fft.rfftn / irfftn, FP32, unnormalised
    inverse) on the same grids: ms per 3D R2C and C2R, and ms of each of our
    passes alone.  CUDA events on the current stream, after warm-up."""
    import torch

    from kwave import _lib

    def timed(fn):
        for _ in range(warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = []
    for nx, ny, nz in grids:
        plan = _lib.Fft3d(nx, ny, nz)
        x = torch.randn((nz, ny, nx), device="cuda", dtype=torch.float32)
        spec = torch.zeros((nz, ny, plan.nxp), device="cuda", dtype=torch.complex64)
        back = torch.empty_like(x)
        st = torch.cuda.current_stream().cuda_stream
        X = torch.fft.rfftn(x)
        row = {"grid": [nx, ny, nz],
               "cufft_r2c_ms": timed(lambda: torch.fft.rfftn(x)),
               "cufft_c2r_ms": timed(lambda: torch.fft.irfftn(X, s=(nz, ny, nx), norm="forward")),
               "own_r2c_ms": timed(lambda: plan.exec(x.data_ptr(), spec.data_ptr(), False, 7, st)),
               "own_c2r_ms": timed(lambda: plan.exec(back.data_ptr(), spec.data_ptr(), True, 7, st))}
        row["own_pass_ms"] = {name: timed(lambda b=bit: plan.exec(x.data_ptr(), spec.data_ptr(), False, b, st))
                              for name, bit in (("x_r2c", 1), ("y", 2), ("z", 4))}
        plan.check()
        plan.close()
        row["own_vs_cufft_r2c"] = row["cufft_r2c_ms"] / row["own_r2c_ms"]
        row["own_vs_cufft_c2r"] = row["cufft_c2r_ms"] / row["own_c2r_ms"]
        out.append(row)
    return {"grids": out,
            "note": "own = the solver's passes run bare (kw_fft3d; in the time loop they are fused with the "
                    "physics); cufft = torch.fft.rfftn / irfftn (norm='forward', unnormalised inverse); "
                    "own_vs_cufft > 1 means the own transform is faster"}


def run_reference(args):
    """The reference arm: the reference algorithm on the host cores (the
    oracle port, numpy + scipy.fft on every host thread), the same workload,
    metric and config as the GPU arm.  `--warmup` untimed time steps, then up
    to `--steps` timed ones, stopping early once the timed steps pass
    REF_TIMED_S seconds (the steps actually timed are reported)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    inp, record, start = build_input(args.n, args.nt)
    from oracle.kspace_oracle import simulate

    npts = args.n ** 3
    w, k_req = max(0, args.warmup), max(1, args.steps)
    stamps = []
    t0 = time.perf_counter()
    REF_TIMED_S = 180.0

    a = max(w, 1) - 1  # stamps[a] closes the last untimed step (one anchoring step when --warmup 0)

    def on_step(t):
        stamps.append(time.perf_counter())
        if len(stamps) - 1 - a >= 1 and stamps[-1] - stamps[a] > REF_TIMED_S:
            raise _SampleDone()

    try:
        simulate(inp, record=record, dtype=np.float32, workers=-1, max_steps=a + 1 + k_req, on_step=on_step)
    except _SampleDone:
        pass
    k = len(stamps) - 1 - a
    per = (stamps[-1] - stamps[a]) / k
    value = npts / per
    cores = os.cpu_count()
    so = mapped_repo_libraries()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": k, "warmup": w, "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config((args.n,) * 3, args.nt, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"time steps {a + 2}..{a + 1 + k} of the {args.n}^3 run after {a + 1} untimed, "
                                   f"numpy/scipy.fft workers={cores}; MATLAB reference not installable here"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "repo_libraries_mapped": so,
        "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--nt", type=int, default=1200)
    ap.add_argument("--e2e-reps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default=None, help="Nx,Ny,Nz for a smaller profiling case (default n^3)")
    ap.add_argument("--batch-sims", type=int, default=48, help="simulations in the batched sample (0: skip)")
    ap.add_argument("--batch-nt", type=int, default=500, help="time steps of each batched simulation")
    ap.add_argument("--serve-requests", type=int, default=16, help="requests in the served sample (0: skip)")
    ap.add_argument("--no-tune", action="store_true", help="keep the built-in launch schedule (no kw_tune)")
    ap.add_argument("--no-fft-sample", action="store_true", help="skip the comparison with cuFFT")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    from kwave import _lib

    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else None
    inp, record, start = build_input(args.n, args.nt, shape)
    nt_needed = args.warmup + args.steps
    sess_inp = dict(inp)
    if nt_needed > int(inp["Nt"]):
        sess_inp["Nt"] = nt_needed
    pinned = pin_inputs(sess_inp)
    npts = int(inp["Nx"]) * int(inp["Ny"]) * int(inp["Nz"])

    # ----- launch schedule: timed once by kw_tune before anything is measured
    # and remembered for this grid, like an FFT plan; the session and the
    # solves below use it -----
    sched = None
    if not args.no_tune:
        t0 = time.perf_counter()
        sched = _lib.tune(pinned, record=record, start_index=start, device=local)
        sched["tune_s"] = time.perf_counter() - t0

    # ----- device-resident timing -----
    sess = _lib.Session(pinned, record=record, start_index=start, device=local)
    sched_used = sess.schedule
    sess.advance(args.warmup)
    sess.sync()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    sess.advance(args.steps)
    ms = sess.elapsed_ms()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches_per_step = sess.launches_per_step
    sess.close()
    value, ms_max = replica_throughput(ms, npts * args.steps, dist, device="cuda")
    ms_per_step = ms_max / args.steps

    # ----- end to end: a whole solve through kw_solve from pinned host memory -----
    e2e_inp = pin_inputs(inp)
    e2e_vals = []
    d2h = npts * 4 * sum(1 for r in record if r in ("p_max", "p_rms", "p_min"))
    for _ in range(args.e2e_reps):
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.solve(e2e_inp, record=record, start_index=start, device=local)
        torch.cuda.synchronize()
        dt_e2e = time.perf_counter() - t0
        t_t = torch.tensor([dt_e2e], device="cuda")
        if dist is not None:
            dist.all_reduce(t_t, op=dist.ReduceOp.MAX)
        e2e_vals.append(world * npts * int(inp["Nt"]) / float(t_t.item()))
    e2e_value = max(e2e_vals) if e2e_vals else None

    peak, peak_kind = peaks()
    achieved = B_ALG * npts / (ms_per_step / 1e3) / 1e9
    traffic = traffic_per_step(args.n) if not args.shape else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config((inp["Nx"], inp["Ny"], inp["Nz"]), inp["Nt"], world),
        "schedule": {"used": {k: sched_used[k] for k in ("slab_planes", "streams", "row_lines", "col_lines")},
                     "tuned": sched},
        "e2e": ({"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_bytes(inp), "d2h_bytes_per_step": d2h,
                 "note": f"one e2e step = one whole {int(inp['Nt'])}-step solve via kw_solve, pinned host buffers"
                         + ("; launch schedule tuned once beforehand (kw_tune, schedule.tuned.tune_s)"
                            if sched else "")}
                if e2e_value else None),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "unit_of_work": f"one time step ({B_ALG:.0f} B algorithmic per grid point)"},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, per, w, k = cpu_sample(inp, record)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                "sample": f"time steps {w + 1}..{w + k} of the same {args.n}^3 run, oracle "
                                          f"(numpy/scipy.fft, all host threads), {per:.2f} s/step, "
                                          f"{per * k:.1f} s timed"}
    if rank == 0 and world == 1 and not args.shape:
        if not args.no_fft_sample:
            line["fft_vs_cufft"] = fft_sample()
        if args.batch_sims > 0:
            line["batched"] = batched_sample(args.batch_sims, args.batch_nt)
        if args.serve_requests > 0:
            line["served"] = served_sample(args.serve_requests)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
