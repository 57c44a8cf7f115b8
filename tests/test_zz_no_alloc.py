"""kw_kspace_gradient_noalloc through the C ABI, against kw_solve.

With an initial pressure p0 and a sensor on every grid point, the particle
velocity kw_solve records at the first time step is
    ux = dt / rho0 * gx / 2,   uy = dt / rho0 * gy / 2
(kspaceFirstOrder2D.m:920-921), where (gx, gy) is the k-space staggered
gradient of p0 that kw_kspace_gradient_noalloc computes from caller-owned
device buffers.  Two calls in a row must each match it.  This file is named
to be collected last, so the entry point also runs after everything else the
suite has done on the device; it passes alone in a fresh process as well.
"""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative L2 error, FP32 spectral operators computed two ways


def _case(n, seed):
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, smooth

    rng = np.random.default_rng(seed)
    kg = KWaveGrid(n, (1e-4, 1.2e-4))
    kg.set_time(2, 0.3e-4 / 1500)
    p0 = smooth(rng.standard_normal(n), True)
    inp, record, start, meta = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": p0},
                                       {"mask": np.ones(n), "record": ["u"]}, pml_size=6, smooth_p0=False)
    return inp


def _gradient_from_solve(inp):
    """(gx, gy) as [ny][nx] arrays from the velocity kw_solve records at t = 1."""
    from kwave import _lib

    out = _lib.solve(inp, ("u",))
    nx, ny = int(inp["Nx"]), int(inp["Ny"])
    scale = 2.0 * float(np.asarray(inp["rho0"]).reshape(-1)[0]) / float(inp["dt"])
    return [scale * out[k][:, 0].reshape(ny, nx) for k in ("ux", "uy")]


def _noalloc(inp, d_f, d_gx, d_gy):
    import torch
    from kwave import _lib

    _lib.kspace_gradient_noalloc(d_f.data_ptr(), d_gx.data_ptr(), None if d_gy is None else d_gy.data_ptr(),
                                 int(inp["Nx"]), int(inp["Ny"]), inp["dx"], inp["dy"], inp["c_ref"], inp["dt"],
                                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [(64, 48), (45, 60)])
def test_gradient_noalloc_matches_solve_twice(n):
    import torch

    inp = _case(n, seed=sum(n))
    want_x, want_y = _gradient_from_solve(inp)
    nx, ny = n
    f = np.asarray(inp["p0_source_input"], np.float32).reshape(nx, ny).T.copy()  # [ny][nx], x fastest
    d_f = torch.from_numpy(f).cuda()
    results = []
    for _ in range(2):
        d_gx = torch.full_like(d_f, float("nan"))
        d_gy = torch.full_like(d_f, float("nan"))
        _noalloc(inp, d_f, d_gx, d_gy)
        gx, gy = d_gx.cpu().numpy(), d_gy.cpu().numpy()
        assert np.isfinite(gx).all() and np.isfinite(gy).all()
        assert rel_l2(gx, want_x) < TOL, rel_l2(gx, want_x)
        assert rel_l2(gy, want_y) < TOL, rel_l2(gy, want_y)
        results.append((gx, gy))
    np.testing.assert_array_equal(results[0][0], results[1][0])
    np.testing.assert_array_equal(results[0][1], results[1][1])


def test_gradient_noalloc_x_only():
    import torch

    inp = _case((50, 36), seed=5)
    want_x, _ = _gradient_from_solve(inp)
    f = np.asarray(inp["p0_source_input"], np.float32).reshape(50, 36).T.copy()
    d_f = torch.from_numpy(f).cuda()
    d_gx = torch.empty_like(d_f)
    _noalloc(inp, d_f, d_gx, None)
    assert rel_l2(d_gx.cpu().numpy(), want_x) < TOL


def test_gradient_noalloc_rejects_what_it_cannot_hold():
    import torch
    from kwave import _lib

    d = torch.zeros(16, device="cuda")
    args = (1e-4, 1e-4, 1500.0, 1e-8)
    with pytest.raises(_lib.KwaveError) as e:
        _lib.kspace_gradient_noalloc(d.data_ptr(), d.data_ptr(), None, 2048, 4, *args)
    assert e.value.code == _lib.KW_ERR_INVALID_ARGUMENT and "1024" in str(e.value)
    with pytest.raises(_lib.KwaveError) as e:
        _lib.kspace_gradient_noalloc(d.data_ptr(), d.data_ptr(), None, 4, 11, *args)
    assert e.value.code == _lib.KW_ERR_UNSUPPORTED
    host = np.zeros(16, np.float32)
    with pytest.raises(_lib.KwaveError) as e:
        _lib.kspace_gradient_noalloc(host.ctypes.data, d.data_ptr(), None, 4, 4, *args)
    assert e.value.code == _lib.KW_ERR_INVALID_ARGUMENT and "device" in str(e.value)
