"""The transform-length tables the build instantiates kernels for.

ct_sizes.h lists the compile-time FFT lengths (one generated translation unit
each), tma_sizes.h the lengths of the TMA-fed column passes (one generated
unit each for the fused last-axis operator).  Every TMA length must also be a
compile-time length (the TMA kernels run the compile-time engine), and no TMA
length may exceed 256 (a tensor copy's box holds at most 256 elements along a
dimension).
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "k-wave_b200"))

import build  # noqa: E402  (k-wave_b200/build.py)


def _five_smooth(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def test_compile_time_lengths_are_every_five_smooth_length_64_to_1024():
    ct = build.ct_sizes()
    assert ct == sorted(set(ct))
    assert ct == [n for n in range(64, 1025) if _five_smooth(n)]
    assert len(ct) == 61


def test_tma_lengths_are_compile_time_lengths_up_to_256():
    ct = set(build.ct_sizes())
    tma = build.tma_sizes()
    assert tma == sorted(set(tma))
    assert tma == [n for n in range(64, 257) if _five_smooth(n)]
    assert set(tma) <= ct
