"""GPU outputs against the FP64 and FP32 oracle on the measured configurations.

* The benchmarked 256^3 heterogeneous absorbing nonlinear workload (TMA
  y pass and fused last-axis kernels of length 256, the two-z-slab chains on
  two streams, the k-space corrected additive plane source), run three ways:
  kw_solve with the built-in schedule, kw_solve after kw_tune picked one,
  and a session advanced in chunks.
* The FP64-check configuration: 128^3 two-ball lossless medium with a
  200-point Cartesian sphere sensor.

Each test asserts the relative L2 bar (1e-4; 1e-5 for the linear lossless
case).  With KWAVE_B200_ACCURACY_REPORT=<file.md> set, it also writes the
per-output error table (GPU FP32 against FP64, the FP32 oracle against FP64
for scale); KWAVE_B200_ACCURACY_NT=<n> sets the number of time steps.
"""
import os
import time

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _errors(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return rel_l2(a, b), float(np.max(np.abs(a - b))), float(np.max(np.abs(b)))


def _report(title, lines_head, runs, o64, o32, keys):
    path = os.environ.get("KWAVE_B200_ACCURACY_REPORT")
    if not path:
        return
    cols = list(runs)
    out = [f"# {title}", ""] + lines_head + [
        "",
        "| output | " + " | ".join(f"GPU ({c}) vs FP64: rel. L2 | max abs" for c in cols)
        + " | FP32 oracle vs FP64: rel. L2 | max abs | max abs value |",
        "|---|" + "---|---|" * len(cols) + "---|---|---|"]
    for k in keys:
        cells = []
        for c in cols:
            g, mg, _ = _errors(runs[c][k], o64[k])
            cells.append(f"{g:.2e} | {mg:.2e}")
        c32, m32, ref = _errors(o32[k], o64[k])
        out.append(f"| {k} | " + " | ".join(cells) + f" | {c32:.2e} | {m32:.2e} | {ref:.3e} |")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def _oracles(inp, record, start):
    from oracle.kspace_oracle import simulate

    t0 = time.perf_counter()
    o64 = simulate(inp, record=record, record_start_index=start, dtype=np.float64)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    o32 = simulate(inp, record=record, record_start_index=start, dtype=np.float32)
    t32 = time.perf_counter() - t0
    return o64, o32, t64, t32


def test_headline_256_cubed_against_the_oracle():
    from kwave import _lib
    from kwave.simulation import prepare
    from kwave.workloads import het_absorbing_3d

    nt = int(os.environ.get("KWAVE_B200_ACCURACY_NT", "12"))
    kg, medium, source, sensor = het_absorbing_3d(n=256, nt=nt, record=("p_max", "p_rms", "p_final"))
    inp, record, start, _ = prepare(kg, medium, source, sensor)
    runs, times = {}, {}
    try:
        _lib.wisdom_forget()
        t0 = time.perf_counter()
        runs["built-in schedule"] = _lib.solve(inp, record=record, start_index=start, device=0)
        times["built-in schedule"] = time.perf_counter() - t0
        sched = _lib.tune(inp, record=record, start_index=start, device=0)
        runs["tuned schedule"] = _lib.solve(inp, record=record, start_index=start, device=0)
        s = _lib.Session(inp, record=record, start_index=start, device=0)
        try:
            done = 0
            for chunk in (5, 1, nt):
                m = min(chunk, nt - done)
                if m > 0:
                    s.advance(m)
                    done += m
            s.sync()
            runs["session"] = s.read()
        finally:
            s.close()
    finally:
        _lib.wisdom_forget()
    o64, o32, t64, t32 = _oracles(inp, record, start)
    keys = ["p_max", "p_rms", "p_final"]
    for name, out in runs.items():
        for k in keys:
            assert rel_l2(out[k], o64[k]) <= 1e-4, (name, k, "fp64")
            assert rel_l2(out[k], o32[k]) <= 1e-4, (name, k, "fp32")
    _report(f"Accuracy against the FP64 oracle: 256^3 heterogeneous absorbing nonlinear workload, Nt {nt}",
            ["Command (one B200; the oracle runs on the host's threads):", "", "```",
             f"KWAVE_B200_ACCURACY_NT={nt} KWAVE_B200_ACCURACY_REPORT=<file> "
             "python -m pytest tests/test_gpu_accuracy.py -m gpu -k headline", "```", "",
             "The benchmarked workload (c = 1500 + 60 z, rho = 1000 + 50 z' smoothed unit-std noise, "
             "alpha 0.75 dB/(MHz^y cm), y 1.5, B/A 6, 48 x 48 additive plane pressure source, "
             "1 MHz 3-cycle tone burst of 1 MPa, every grid point a sensor), first "
             f"{nt} time steps (the source is active throughout).  Reference = the oracle in FP64 (the "
             "reference algorithm with DataCast 'off'); the FP32 oracle is the same algorithm in single "
             "precision (complex64 FFTs), for scale.",
             f"Schedule after kw_tune: {sched.get('slab_planes')} z planes per slab, "
             f"{sched.get('streams')} stream(s).",
             f"Run times: GPU solve {times['built-in schedule']:.2f} s (set-up included), FP64 oracle "
             f"{t64:.0f} s, FP32 oracle {t32:.0f} s."], runs, o64, o32, keys)


def test_two_ball_128_cubed_against_the_oracle():
    from kwave import _lib
    from kwave.simulation import prepare
    from kwave.workloads import two_ball_3d

    nt = int(os.environ.get("KWAVE_B200_ACCURACY_NT", "60"))
    kg, medium, source, sensor = two_ball_3d(n=128, nt=nt)
    inp, record, start, _ = prepare(kg, medium, source, sensor)
    t0 = time.perf_counter()
    gpu = _lib.solve(inp, record=record, start_index=start, device=0)
    t_gpu = time.perf_counter() - t0
    o64, o32, t64, t32 = _oracles(inp, record, start)
    keys = [k for k in ("p", "ux", "uy", "uz", "p_max", "p_rms") if k in gpu and k in o64]
    for k in keys:
        assert rel_l2(gpu[k], o64[k]) <= 1e-5, k  # linear lossless
    _report(f"Accuracy against the FP64 oracle: 128^3 two-ball configuration, Nt {nt}",
            ["Command (one B200; the oracle runs on the host's threads):", "", "```",
             f"KWAVE_B200_ACCURACY_NT={nt} KWAVE_B200_ACCURACY_REPORT=<file> "
             "python -m pytest tests/test_gpu_accuracy.py -m gpu -k two_ball", "```", "",
             "3D 128^3 homogeneous lossless medium (c 1500 m/s, rho 1000 kg/m^3, dx 0.1 mm), initial "
             "pressure 5 ball(64,64,64, r 5) + 3 ball(40,80,64, r 3) smoothed, sensor = a 200-point "
             "Cartesian sphere of radius 4 mm mapped to the nearest grid points, records p, u, p_max, "
             "p_rms, CFL 0.3.  Reference = the oracle in FP64 (the reference algorithm with DataCast "
             "'off'); the FP32 oracle is the same algorithm in single precision, for scale.",
             f"Run times: GPU solve {t_gpu:.2f} s (set-up included), FP64 oracle {t64:.0f} s, "
             f"FP32 oracle {t32:.0f} s."], {"FP32": gpu}, o64, o32, keys)
