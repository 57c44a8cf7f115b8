"""The MEX shim (k-wave_b200/mex/kspaceFirstOrderB200_mex.c) compiles
against the C ABI header and a stand-in mex.h with every warning an error,
and fills every kw_input field the input file can carry."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "k-wave_b200", "mex", "kspaceFirstOrderB200_mex.c")
HEADER = os.path.join(ROOT, "include", "kwave_b200.h")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc absent")
@pytest.mark.parametrize("std", ["c99", "c11"])
def test_shim_compiles_against_the_header(std):
    r = subprocess.run(["gcc", f"-std={std}", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tests", "mex_stub"), SHIM],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_shim_sets_every_input_field():
    src = open(SHIM).read()
    hdr = open(HEADER).read()
    body = hdr[hdr.index("/* grid: Nz = 1"):hdr.index("} kw_input;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = set()
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        for part in decl.split(","):  # the last identifier of each declarator
            ids = re.findall(r"[A-Za-z_][A-Za-z0-9_]*", part)
            if ids:
                fields.add(ids[-1])
    assert len(fields) > 50
    missing = sorted(f for f in fields if f"in->{f}" not in src)
    assert not missing, missing


def test_shim_returns_every_output_the_wrapper_reads():
    src = open(SHIM).read()
    for name in ("p", "p_max", "p_min", "p_rms", "p_max_all", "p_min_all", "p_final", "ux", "uy", "uz",
                 "ux_max", "ux_min", "ux_rms", "ux_max_all", "ux_min_all", "ux_final", "ux_non_staggered",
                 "uz_non_staggered", "Nx", "Ny", "Nz", "pml_x_size", "pml_y_size", "pml_z_size"):
        assert f'"{name}"' in src, name
