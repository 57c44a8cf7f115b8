"""The blocked sum of squares behind p_rms / u_rms, restated in numpy FP32.

The step kernels keep, per sensor point, a plain FP32 partial sum of the
squares of the current block of kRmsBlock recorded steps (kernels.cuh) and
add it at the block's end to a Kahan-compensated total; the final rms adds a
still-open block's partial sum.  This restatement follows the device code
step for step (rms_put / rms_store4 in kernels_impl.cuh, k_rms_final in
kernels.cu) and checks the rounding it claims: close to kRmsBlock ulp of the
sum, no worse than a plain FP32 running sum and well inside the 1e-4 bar.
"""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _block():
    with open(os.path.join(ROOT, "k-wave_b200", "csrc", "kernels.cuh")) as f:
        return int(re.search(r"constexpr int kRmsBlock = (\d+);", f.read()).group(1))


def _blocked_sum(p, B):
    """Sum of squares over axis 0 as the device accumulates it (FP32)."""
    f32 = np.float32
    acc = np.zeros((2,) + p.shape[1:], f32)  # Kahan {sum, compensation}
    blk = np.zeros(p.shape[1:], f32)
    for fi in range(1, p.shape[0] + 1):
        v = p[fi - 1].astype(f32)
        j = (fi - 1) % B
        v64 = v.astype(np.float64)  # v * v is exact in FP64: one rounding, as the device's fma
        b = (v64 * v64).astype(f32) if j == 0 else (blk.astype(np.float64) + v64 * v64).astype(f32)
        if j == B - 1:
            if fi == B:
                acc[:] = 0
            y = (b - acc[1]).astype(f32)
            t = (acc[0] + y).astype(f32)
            acc[1] = ((t - acc[0]) - y).astype(f32)
            acc[0] = t
        else:
            blk = b
    partial = (p.shape[0] % B) != 0
    return (acc[0] + (blk if partial else 0)).astype(f32)


def _plain_sum(p):
    s = np.zeros(p.shape[1:], np.float32)
    for v in p.astype(np.float32):
        s = (s + v * v).astype(np.float32)
    return s


def test_blocked_sum_of_squares_rounding():
    B = _block()
    rng = np.random.default_rng(3)
    for nt in (B - 3, B, 5 * B + 7, 1200):  # open block, one block, several, the 256^3 workload's Nt
        t = np.arange(nt)[:, None]
        p = (1e5 * np.sin(0.05 * t + rng.uniform(0, 6.3, (1, 4000)))
             * (1 + 0.3 * rng.standard_normal((nt, 4000)))).astype(np.float32)
        exact = np.sum(p.astype(np.float64) ** 2, axis=0)
        blocked = _blocked_sum(p, B).astype(np.float64)
        plain = _plain_sum(p).astype(np.float64)
        err_b = np.abs(blocked - exact) / exact
        err_p = np.abs(plain - exact) / exact
        ulp = np.finfo(np.float32).eps
        assert err_b.max() <= (B + 2) * ulp, (nt, err_b.max() / ulp)  # the worst-case bound
        assert err_b.mean() <= ulp, (nt, err_b.mean() / ulp)  # typical: below one ulp
        assert err_b.mean() <= err_p.mean() + 0.1 * ulp, nt  # never worse than a plain running sum
        rms = np.sqrt(blocked / nt)
        assert np.max(np.abs(rms - np.sqrt(exact / nt)) / np.sqrt(exact / nt)) <= 1e-5
