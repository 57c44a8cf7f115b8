"""The file drop-in on the GPU: a k-Wave v1.2 input file (the layout
kspaceFirstOrder_saveToDisk.m writes) run through kw_run_file and through the
solver binary's command line gives the same sensor data, bit for bit, as the
in-memory kw_solve, in the output layout kspaceFirstOrder3DC.m:569-776 reads."""
import os
import subprocess

import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "k-wave_b200", "kspaceFirstOrder-B200")


def _same(a, b):
    assert set(a) == set(b), (sorted(a), sorted(b))
    for k in a:
        assert a[k].shape == b[k].shape, k
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_run_file_3d_matches_solve(tmp_path):
    from kwave import _lib, h5io

    record = ("p", "p_max", "p_min", "p_rms", "u", "u_max", "p_final", "u_final", "p_max_all")
    inp, _, start, meta = case_3d_het(n=(36, 30, 32), nt=50, record=record)
    fin, fout = tmp_path / "in.h5", tmp_path / "out.h5"
    h5io.write_input_file(fin, inp)
    _lib.run_file(fin, fout, record, start_index=7)
    got = h5io.read_output_file(fout, 3)
    want = _lib.solve(inp, record, start_index=7)
    _same(got, want)
    with h5io.File(fout) as f:
        a = f.attrs("/")
        assert a["file_type"] == "output" and a["major_version"] == "1" and a["minor_version"] == "2"
        assert int(f.read("/Nx").reshape(-1)[0]) == 36
        assert f.read("/Nx").shape == (1, 1, 1) and f.read("/Nx").dtype == np.uint64
        assert int(f.read("/pml_z_size").reshape(-1)[0]) == int(inp["pml_z_size"])
        assert f.read("/p").shape == (1, 50 - 7 + 1, want["p"].shape[0])
        assert f.read("/p_final").shape == (32, 30, 36)


def test_command_line_2d_matches_solve(tmp_path):
    from kwave import _lib, h5io

    inp, _, start, meta = case_2d_p0(n=(48, 40), nt=40)
    fin, fout = tmp_path / "in.h5", tmp_path / "out.h5"
    h5io.write_input_file(fin, inp)
    r = subprocess.run([BIN, "-i", str(fin), "-o", str(fout), "--p_raw", "--u_rms", "--p_min_all", "-s", "3",
                        "-t", "4", "--verbose", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = h5io.read_output_file(fout, 2)
    want = _lib.solve(inp, ("p", "u_rms", "p_min_all"), start_index=3)
    _same(got, want)
    with h5io.File(fout) as f:
        names = f.children(f.root)
        assert "pml_z_size" not in names and "uz_rms" not in names


def test_command_line_default_records_p(tmp_path):
    from kwave import _lib, h5io

    inp, _, start, meta = case_2d_p0(n=(32, 36), nt=20)
    fin, fout = tmp_path / "in.h5", tmp_path / "out.h5"
    h5io.write_input_file(fin, inp)
    assert _lib.cli_main(["kspaceFirstOrder-B200", "-i", str(fin), "-o", str(fout)]) == 0
    got = h5io.read_output_file(fout, 2)
    assert set(got) == {"p"}
    np.testing.assert_array_equal(got["p"], _lib.solve(inp, ("p",))["p"])


def test_cuboid_outputs_are_groups(tmp_path):
    """Cuboid sensors: one dataset per cuboid under /<output>/<k>, MATLAB
    order [x, y, z, t] (kspaceFirstOrder3DC.m:651-700)."""
    from kwave import _lib, h5io
    from kwave.simulation import prepare
    from kwave.utils import KWaveGrid, make_ball

    n = (30, 32, 36)
    kg = KWaveGrid(n, (1e-4, 1e-4, 1e-4))
    kg.set_time(30, 0.3e-4 / 1500)
    corners = np.array([[4, 5, 6, 10, 12, 9], [20, 18, 25, 24, 22, 30]]).T
    rec = ("p", "p_max")
    inp, _, _, _ = prepare(kg, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": make_ball(*n, 15, 16, 18, 3)},
                           {"mask": corners, "record": list(rec)}, pml_size=5)
    fin, fout = tmp_path / "in.h5", tmp_path / "out.h5"
    h5io.write_input_file(fin, inp)
    _lib.run_file(fin, fout, rec)
    got = h5io.read_output_file(fout, 3)
    flat = _lib.solve(inp, rec)
    start = 0
    for k in range(corners.shape[1]):
        x1, y1, z1, x2, y2, z2 = corners[:, k]
        shape = (x2 - x1 + 1, y2 - y1 + 1, z2 - z1 + 1)
        npts = int(np.prod(shape))
        p = got["p"][k]
        assert p.shape == shape + (30,)
        np.testing.assert_array_equal(p.reshape(npts, 30, order="F"), flat["p"][start:start + npts])
        np.testing.assert_array_equal(got["p_max"][k].reshape(-1, order="F"), flat["p_max"][start:start + npts])
        start += npts
