"""Per-output error of the GPU solver against the FP64 oracle on the FP64-check
configuration: 3D 128^3 homogeneous lossless medium, initial pressure from two
smoothed balls, a 200-point Cartesian sphere sensor mapped to the grid,
record {p, u, p_max, p_rms}, Nt 600.  The FP32 oracle (the reference's
single-precision path restated) is reported beside it for scale.

Run on a machine with a GPU (a few minutes: the oracle is numpy):
    python tests/accuracy_report.py [--n 128] [--nt 600] [--out report.md]
Test infrastructure: it executes the oracle as the checker only.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "k-wave_b200"))
sys.path.insert(0, ROOT)


def errors(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    num = np.linalg.norm((a - b).ravel())
    den = np.linalg.norm(b.ravel())
    return (num / den if den else float(num)), float(np.max(np.abs(a - b))), float(np.max(np.abs(b)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--nt", type=int, default=600)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    from kwave import _lib
    from kwave.simulation import prepare
    from kwave.workloads import two_ball_3d
    from oracle.kspace_oracle import simulate

    kg, medium, source, sensor = two_ball_3d(n=args.n, nt=args.nt)
    inp, record, start, meta = prepare(kg, medium, source, sensor)
    t0 = time.perf_counter()
    gpu = _lib.solve(inp, record=record, start_index=start)
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    o64 = simulate(inp, record=record, record_start_index=start, dtype=np.float64)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    o32 = simulate(inp, record=record, record_start_index=start, dtype=np.float32)
    t32 = time.perf_counter() - t0

    keys = [k for k in ("p", "ux", "uy", "uz", "p_max", "p_rms") if k in gpu and k in o64]
    lines = [f"Configuration: {args.n}^3, Nt {args.nt}, {len(inp['sensor_mask_index'])} sensor points; "
             f"records {', '.join(record)}.",
             f"Run times: GPU solve {t_gpu:.2f} s (including set-up), FP64 oracle {t64:.0f} s, "
             f"FP32 oracle {t32:.0f} s (numpy / scipy.fft, all host threads).", "",
             "| output | GPU FP32 vs FP64: rel. L2 | max abs | FP32 oracle vs FP64: rel. L2 | max abs | max abs value |",
             "|---|---|---|---|---|---|"]
    for k in keys:
        g, mg, ref = errors(gpu[k], o64[k])
        c, mc, _ = errors(o32[k], o64[k])
        lines.append(f"| {k} | {g:.2e} | {mg:.2e} | {c:.2e} | {mc:.2e} | {ref:.3e} |")
    text = "\n".join(lines)
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
