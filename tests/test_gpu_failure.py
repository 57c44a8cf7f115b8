"""Failure detection on the GPU: a bounded wait that runs out.

Every mbarrier wait of the TMA-fed kernels (the y pass and the fused
last-axis operator) has a time limit.  The test hook
KWAVE_B200_TEST_SKIP_TMA_TILE makes one tile's load be announced on its
barrier but never issued, so that wait can only end by running out; nothing
else is in flight for it, and the GPU is never faulted.  The kernel must then
leave its loop, drain its other copies and return; the session reports
KW_ERR_CUDA promptly; and the device stays usable for an ordinary solve.
"""
import time

import numpy as np
import pytest

from helpers import case_3d_het, oracle_outputs, rel_l2

pytestmark = pytest.mark.gpu


def test_tma_wait_that_runs_out_ends_the_kernel_and_reports_it(monkeypatch):
    from kwave import _lib

    # 64 x 72 x 64: the y pass (72) and the last-axis operator (64) both run on TMA
    inp, record, start, _ = case_3d_het(n=(64, 72, 64), nt=12, record=("p", "p_max"))
    monkeypatch.setenv("KWAVE_B200_TMA_WAIT_US", "100")
    monkeypatch.setenv("KWAVE_B200_TEST_SKIP_TMA_TILE", "0")
    s = _lib.Session(inp, record=record, start_index=start, device=0)
    monkeypatch.delenv("KWAVE_B200_TEST_SKIP_TMA_TILE")
    monkeypatch.delenv("KWAVE_B200_TMA_WAIT_US")
    try:
        t0 = time.perf_counter()
        s.advance(6)
        with pytest.raises(_lib.KwaveError) as e:
            s.sync()
        waited = time.perf_counter() - t0
    finally:
        s.close()
    assert e.value.code == _lib.KW_ERR_CUDA
    assert "timed out" in str(e.value)
    # each hooked launch gives up after 100 us: the six steps end in well under
    # a second, not after the default 2 s limit per wait
    assert waited < 1.5, waited

    # the context is intact: an ordinary solve on the same device is correct
    gpu = _lib.solve(inp, record=record, start_index=start, device=0)
    ora = oracle_outputs(inp, record, start, dtype=np.float64)
    for k in ("p", "p_max"):
        assert rel_l2(gpu[k], ora[k]) <= 1e-4, k
