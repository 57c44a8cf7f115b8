"""Seeded synthetic simulation inputs.

No public benchmark suite is involved: the workloads are the reference's
own example-style setups with the shapes, sizes and value distributions of
the measured configurations, generated from fixed seeds.  Each builder
returns ``(kgrid, medium, source, sensor)`` for ``kspace_first_order`` /
``prepare``.
"""
from __future__ import annotations

import numpy as np

from .utils import KWaveGrid, make_ball, make_cart_circle, make_cart_sphere, make_disc, tone_burst


def smoothed_noise(shape, seed, sigma=4.0):
    """White N(0,1) noise, Gaussian-filtered (periodic), renormalised to unit std."""
    from scipy.ndimage import gaussian_filter

    z = np.random.default_rng(seed).standard_normal(shape)
    z = gaussian_filter(z, sigma=sigma, mode="wrap")
    return (z - z.mean()) / z.std()


def two_disc_2d(n=128, dx=1e-4, t_end=8e-6, cart_points=50, cart_radius=4e-3):
    """2D homogeneous lossless medium, initial pressure from two smoothed
    discs, Cartesian circle of sensor points (mapped to the nearest grid
    points, as the file-based path requires)."""
    kgrid = KWaveGrid((n, n), (dx, dx))
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    p0 = 5 * make_disc(n, n, n // 2, n // 2, 5) + 3 * make_disc(n, n, n * 40 // 128, n * 80 // 128, 3)
    kgrid.make_time(1500.0, 0.3, t_end)
    source = {"p0": p0}
    sensor = {"mask": make_cart_circle(cart_radius, cart_points), "record": ["p"]}
    return kgrid, medium, source, sensor


def het_absorbing_3d(n=256, nt=1200, dx=1e-4, pml=10, plane=48, record=("p_max", "p_rms"), shape=None):
    """3D heterogeneous, power-law absorbing, nonlinear medium (c = 1500 + 60 z,
    rho = 1000 + 50 z', z smoothed unit-std noise), an additive plane pressure
    source driven by a 1 MHz 3-cycle tone burst of 1 MPa, and every grid
    point a sensor.  `shape` overrides the n^3 grid (profiling cases)."""
    shape = tuple(shape) if shape else (n, n, n)
    kgrid = KWaveGrid(shape, (dx, dx, dx))
    c = 1500.0 + 60.0 * smoothed_noise(shape, 2)
    rho = 1000.0 + 50.0 * smoothed_noise(shape, 3)
    medium = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
    dt = 0.3 * dx / c.max()
    kgrid.set_time(nt, dt)
    mask = np.zeros(shape)
    p = min(plane, min(shape[1:]) - 2 * pml)
    y0, z0 = (shape[1] - p) // 2, (shape[2] - p) // 2
    mask[pml, y0:y0 + p, z0:z0 + p] = 1
    sig = 1e6 * tone_burst(1.0 / dt, 1e6, 3)
    source = {"p_mask": mask, "p": sig, "p_mode": "additive"}
    sensor = {"mask": np.ones(shape), "record": list(record)}
    return kgrid, medium, source, sensor


def two_ball_3d(n=128, nt=600, dx=1e-4, sphere_points=200, sphere_radius=4e-3,
                record=("p", "u", "p_max", "p_rms")):
    """3D homogeneous lossless medium, initial pressure from two smoothed
    balls, a Cartesian sphere of sensor points mapped to the grid."""
    kgrid = KWaveGrid((n, n, n), (dx, dx, dx))
    medium = {"sound_speed": 1500.0, "density": 1000.0}
    p0 = 5 * make_ball(n, n, n, n // 2, n // 2, n // 2, 5) + \
        3 * make_ball(n, n, n, n * 40 // 128, n * 80 // 128, n // 2, 3)
    kgrid.set_time(nt, 0.3 * dx / 1500.0)
    source = {"p0": p0}
    sensor = {"mask": make_cart_sphere(sphere_radius, sphere_points), "record": list(record)}
    return kgrid, medium, source, sensor


EDGE_SIZES = (64, 72, 75, 80, 81, 90, 96, 100, 108, 120, 125, 128, 135, 144, 150, 160, 162, 180, 192)


def uneven_lossy_3d(index, n_sims=48, nt=500, dx=1e-4, n_sensors=200, seed=4):
    """One member of a batch of independent 3D linear lossy simulations on
    uneven 2^a 3^b 5^c grids: smoothed random media (c in [1400, 1600],
    rho in [950, 1050]), y = 1.1, point or disc initial pressure, random
    sensor points."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice(EDGE_SIZES, size=(n_sims, 3))
    kinds = rng.integers(0, 2, size=n_sims)
    shape = tuple(int(s) for s in sizes[index])
    r2 = np.random.default_rng(seed * 1000 + index)
    zc = smoothed_noise(shape, seed * 1000 + index + 1)
    zr = smoothed_noise(shape, seed * 1000 + index + 2)
    c = 1400 + 200 * (zc - zc.min()) / (zc.max() - zc.min())
    rho = 950 + 100 * (zr - zr.min()) / (zr.max() - zr.min())
    kgrid = KWaveGrid(shape, (dx, dx, dx))
    kgrid.set_time(nt, 0.3 * dx / c.max())
    medium = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.1}
    centre = [int(r2.integers(s // 4, 3 * s // 4)) + 1 for s in shape]
    if kinds[index] == 0:
        p0 = np.zeros(shape)
        p0[tuple(x - 1 for x in centre)] = 1.0
    else:
        p0 = make_ball(*shape, *centre, 3)
    mask = np.zeros(int(np.prod(shape)))
    mask[r2.choice(mask.size, n_sensors, replace=False)] = 1
    sensor = {"mask": mask.reshape(shape, order="F"), "record": ["p"]}
    return kgrid, medium, {"p0": p0}, sensor


def five_smooth(lo, hi):
    """Integers in [lo, hi] with no prime factor above 5 (FFT-friendly edges)."""
    out = []
    for n in range(lo, hi + 1):
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            out.append(n)
    return tuple(out)


EDGES_2D = five_smooth(256, 1024)
EDGES_3D = five_smooth(64, 256)


def served_request(index, seed=5, rate=20.0, dx=1e-4, pml=10, n_sensors=64):
    """The `index`-th request of a seeded Poisson stream (mean `rate` per
    second): arrival time plus (kgrid, medium, source, sensor).  Half are 2D
    (edges 256..1024), half 3D (edges 64..256), all 2^a 3^b 5^c; half
    lossless, half power-law absorbing with y in U[1.0, 1.8] (y = 1 exactly
    is excluded, as the reference rejects it); smoothed random media; a
    plane pressure source driven by a tone burst; Nt in U[300, 1500]."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=index + 1)
    arrival = float(np.cumsum(gaps)[index])
    r = np.random.default_rng(seed * 100003 + index)
    three_d = bool(r.integers(0, 2))
    edges = EDGES_3D if three_d else EDGES_2D
    n = int(r.choice(edges))
    dim = 3 if three_d else 2
    shape = (n,) * dim
    absorbing = bool(r.integers(0, 2))
    alpha_power = float(r.uniform(1.0, 1.8))
    if abs(alpha_power - 1.0) < 1e-3:
        alpha_power = 1.001
    nt = int(r.integers(300, 1501))
    zc = smoothed_noise(shape, seed * 100003 + index + 1)
    zr = smoothed_noise(shape, seed * 100003 + index + 2)
    c = 1500.0 + 40.0 * zc
    rho = 1000.0 + 30.0 * zr
    kgrid = KWaveGrid(shape, (dx,) * dim)
    dt = 0.3 * dx / c.max()
    kgrid.set_time(nt, dt)
    medium = {"sound_speed": c, "density": rho}
    if absorbing:
        medium.update(alpha_coeff=0.75, alpha_power=alpha_power)
    mask = np.zeros(shape)
    if three_d:
        mask[pml + 1, pml:n - pml, pml:n - pml] = 1
    else:
        mask[pml + 1, pml:n - pml] = 1
    source = {"p_mask": mask, "p": 1e5 * tone_burst(1.0 / dt, 1e6, 3), "p_mode": "additive"}
    smask = np.zeros(int(np.prod(shape)))
    smask[r.choice(smask.size, n_sensors, replace=False)] = 1
    sensor = {"mask": smask.reshape(shape, order="F"), "record": ["p"]}
    return arrival, (kgrid, medium, source, sensor)
