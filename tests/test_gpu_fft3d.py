"""The solver's own FFT passes as a plain transform (kw_fft3d_*), against
numpy's FP64 FFT: forward half spectra, the unnormalised inverse, and each
pass alone (x, then y, then z compose to the full transform)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRIDS = [
    (64, 72, 64),    # compile-time x, TMA y pass, TMA z pass
    (90, 75, 48),    # compile-time x (no 4-wide path), TMA y (75), runtime-engine z (48)
    (256, 256, 128),  # the headline edge lengths
    (128, 90, 1),    # 2D
    (50, 42, 28),    # runtime engine on every axis (a factor 7)
]


def _run(nx, ny, nz, f, passes=7):
    import torch

    from kwave import _lib

    plan = _lib.Fft3d(nx, ny, nz)
    dev = torch.device("cuda:0")
    real = torch.from_numpy(f.astype(np.float32)).to(dev)
    spec = torch.zeros((nz, ny, plan.nxp), dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    plan.exec(real.data_ptr(), spec.data_ptr(), inverse=False, passes=passes, stream=stream)
    fwd = spec.cpu().numpy()[..., : nx // 2 + 1].copy()
    back = torch.zeros_like(real)
    plan.exec(back.data_ptr(), spec.data_ptr(), inverse=True, passes=passes, stream=stream)
    torch.cuda.synchronize()
    plan.check()
    plan.close()
    return fwd, back.cpu().numpy()


@pytest.mark.parametrize("shape", GRIDS, ids=lambda s: "x".join(map(str, s)))
def test_forward_and_inverse_against_numpy(shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 7 + ny * 3 + nz)
    f = rng.standard_normal((nz, ny, nx))
    fwd, back = _run(nx, ny, nz, f)
    ref = np.fft.rfftn(f, axes=(0, 1, 2) if nz > 1 else (1, 2))
    if nz == 1:
        ref = ref.reshape(fwd.shape)
    err = np.linalg.norm(fwd - ref) / np.linalg.norm(ref)
    assert err <= 2e-6, err
    n = nx * ny * nz
    err_b = np.linalg.norm(back / n - f) / np.linalg.norm(f)
    assert err_b <= 2e-6, err_b


def test_each_pass_is_its_axis_transform():
    nx, ny, nz = 64, 72, 64
    f = np.random.default_rng(3).standard_normal((nz, ny, nx))
    fx, _ = _run(nx, ny, nz, f, passes=1)  # x alone: the row transform
    ref = np.fft.rfft(f, axis=2)
    assert np.linalg.norm(fx - ref) / np.linalg.norm(ref) <= 2e-6
    fxy, _ = _run(nx, ny, nz, f, passes=3)  # x then y
    ref = np.fft.fft(ref, axis=1)
    assert np.linalg.norm(fxy - ref) / np.linalg.norm(ref) <= 2e-6
