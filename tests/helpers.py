"""Shared test helpers: input builders and error norms."""
import numpy as np

from kwave.simulation import prepare
from kwave.utils import KWaveGrid, make_ball, make_disc, tone_burst


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    if den == 0:
        return float(np.linalg.norm(a.ravel()))
    return float(np.linalg.norm((a - b).ravel()) / den)


def oracle_outputs(inp, record, start=1, dtype=np.float32):
    """Oracle outputs converted to the C-ABI output names / shapes."""
    from oracle.kspace_oracle import simulate

    return simulate(inp, record=record, record_start_index=start, dtype=dtype)


def compare(gpu, ora, keys=None):
    keys = keys or [k for k in ora if k in gpu]
    return {k: rel_l2(gpu[k], ora[k]) for k in keys}


def case_2d_p0(n=(64, 48), nt=80, record=("p", "p_max", "p_min", "p_rms", "u", "p_final", "u_final",
                                          "p_max_all", "p_min_all", "u_max_all", "u_min_all", "u_max",
                                          "u_min", "u_rms")):
    kg = KWaveGrid(n, (1e-4, 1e-4))
    kg.set_time(nt, 0.3 * 1e-4 / 1500)
    p0 = 3 * make_disc(n[0], n[1], n[0] // 2, n[1] // 2, 4)
    mask = np.zeros(n)
    mask[5:n[0] - 5:7, 6:n[1] - 6:5] = 1
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    return prepare(kg, medium, {"p0": p0}, {"mask": mask, "record": list(record)}, pml_size=8)


def case_3d_het(n=(32, 36, 40), nt=60, absorbing=True, nonlinear=True, p_mode="additive", stokes=False,
                record=("p", "p_max", "p_rms", "u", "p_final"), seed=7, many=False):
    rng = np.random.default_rng(seed)
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    c = 1500 + 50 * rng.standard_normal(n)
    rho = 1000 + 40 * rng.standard_normal(n)
    kg.set_time(nt, 0.3 * 1e-4 / c.max())
    medium = {"sound_speed": c, "density": rho}
    if absorbing:
        medium.update(alpha_coeff=0.75, alpha_power=1.5)
        if stokes:
            medium["alpha_mode"] = "stokes"
    if nonlinear:
        medium["BonA"] = 6.0
    mask = np.zeros(n)
    mask[6, 10:20, 12:24] = 1
    sig = 1e5 * tone_burst(1.0 / kg.dt, 2e6, 2)
    if many:
        npts = int(mask.sum())
        sig = sig * (1 + 0.1 * np.arange(npts)[:, None])
    source = {"p_mask": mask, "p": sig, "p_mode": p_mode}
    smask = np.zeros(n)
    smask[::5, ::4, ::6] = 1
    return prepare(kg, medium, source, {"mask": smask, "record": list(record)}, pml_size=6)
