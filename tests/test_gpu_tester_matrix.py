"""Parity on the grids and media of the reference's native-code comparison
harness (k-Wave/testing/kWaveTester/kWaveTester.m:175-275, 1240-1400): the
four grid types (128 x 64 x 32 with the PML inside and outside, 125 x 63 x 35
inside, 115 x 61 x 29 outside -- 135 x 81 x 49 once the PML is added), a
40 mm domain, c0 1540 m/s, rho0 1000 kg/m^3, alpha 0.75 dB/(MHz^y cm) with
y 1.5, B/A 6, heterogeneity x1.3 in a ball of radius 10 at the centre,
CFL 0.1, tone bursts of 0.5 MHz and 5 cycles at 1 MPa.  The harness runs
its cases for 10 us; these run the first steps, against the FP64 oracle at
the lossless / lossy bars."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

GRIDS = {  # type: (N, PML sizes, PML inside)
    1: ((128, 64, 32), (20, 10, 10), True),
    2: ((128, 64, 32), (20, 10, 11), False),
    3: ((125, 63, 35), (20, 10, 10), True),
    4: ((115, 61, 29), (10, 10, 10), False),
}
C0, RHO0, ALPHA0, Y, BONA, SC = 1540.0, 1000.0, 0.75, 1.5, 6.0, 1.3
STRENGTH, F0, CYCLES = 1e6, 0.5e6, 5


def _case(gtype, het, absorbing, nonlinear, source, nt=70, stokes=False):
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_ball, tone_burst

    N, pml, inside = GRIDS[gtype]
    dx = 40e-3 / N[0]
    kg = KWaveGrid(N, (dx, dx, dx))
    ball = make_ball(*N, round(N[0] / 2), round(N[1] / 2), round(N[2] / 2), 10) == 1
    medium = {"sound_speed": np.where(ball, C0 * SC, C0) if het else C0,
              "density": np.where(ball, RHO0 * SC, RHO0) if het else RHO0}
    if nonlinear:
        medium["BonA"] = np.where(ball, BONA * SC, BONA) if het else BONA
    if absorbing:
        medium["alpha_coeff"] = np.where(ball, ALPHA0 * SC, ALPHA0) if het else ALPHA0
        medium["alpha_power"] = 2.0 if stokes else Y
        if stokes:
            medium["alpha_mode"] = "stokes"
    kg.make_time(medium["sound_speed"], cfl=0.1)
    kg.set_time(nt, kg.dt)
    if source == "p0":
        src = {"p0": STRENGTH * make_ball(*N, round(N[0] / 2), round(N[1] / 2), round(N[2] / 2), 5)}
    else:  # a plane patch one point inside the PML (kWaveTester.m:1392-1409)
        mask = np.zeros(N)
        r = 15
        mask[pml[0], round(N[1] / 2) - r:round(N[1] / 2) + r,
             round(N[2] / 2) - round(r / 2):round(N[2] / 2) + round(r / 2)] = 1
        src = {"p_mask": mask, "p": STRENGTH * tone_burst(1 / kg.dt, F0, CYCLES), "p_mode": source}
    smask = np.zeros(N)
    smask[::6, ::5, ::4] = 1
    sensor = {"mask": smask, "record": ["p", "p_max", "p_rms", "u", "p_final", "p_max_all"]}
    return prepare(kg, medium, src, sensor, pml_size=pml, pml_inside=inside)


def _check(case, tol):
    from kwave import _lib
    from kwave.simulation import postprocess
    from oracle.kspace_oracle import simulate

    inp, record, start, meta = case
    gpu = postprocess(_lib.solve(inp, record=record, start_index=start), inp, meta)
    ora = postprocess(simulate(inp, record=record, record_start_index=start, dtype=np.float64), inp, meta)
    errs = {k: rel_l2(gpu[k], ora[k]) for k in ora}
    assert max(errs.values()) <= tol, errs
    assert np.abs(ora["p"]).max() > 0
    return gpu


@pytest.mark.parametrize("gtype", [1, 2, 3, 4])
def test_het_absorbing_nonlinear_p0(gtype):
    gpu = _check(_case(gtype, het=True, absorbing=True, nonlinear=True, source="p0"), 1e-4)
    assert gpu["p_final"].shape == GRIDS[gtype][0]  # cut back to the user's grid when the PML is outside


@pytest.mark.parametrize("gtype,mode", [(1, "additive"), (3, "dirichlet"), (4, "additive-no-correction")])
def test_plane_sources(gtype, mode):
    _check(_case(gtype, het=True, absorbing=True, nonlinear=False, source=mode, stokes=(gtype == 4)), 1e-4)


def test_lossless_homogeneous_pml_outside():
    _check(_case(2, het=False, absorbing=False, nonlinear=False, source="additive"), 1e-5)
