"""The C ABI: the library loads without a GPU, exports every entry point the
header declares, and the ctypes mirror matches the C struct layout."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kwave_b200.h")


def declared_functions():
    src = open(HEADER).read()
    decl = r"^(?:int|void|void\s*\*|const char\s*\*|uint64_t)\s*\**\s*(kw_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, src, re.M)))


def test_library_exports_every_declared_symbol():
    from kwave import _lib

    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(_lib.lib, n), f"{n} is declared in the header but not exported"
    assert set(names) == set(_lib.EXPORTED)


def test_version_string():
    from kwave import _lib

    assert "kwave_b200" in _lib.version()


def _c_layout():
    """sizeof / offsetof of every struct member, from a gcc-compiled probe."""
    structs = {
        "kw_input": [f for f, _ in __import__("kwave._lib", fromlist=["KwInput"]).KwInput._fields_],
        "kw_options": [f for f, _ in __import__("kwave._lib", fromlist=["KwOptions"]).KwOptions._fields_],
        "kw_output": [f for f, _ in __import__("kwave._lib", fromlist=["KwOutput"]).KwOutput._fields_],
        "kw_output_sizes": [f for f, _ in __import__("kwave._lib", fromlist=["KwOutputSizes"]).KwOutputSizes._fields_],
        "kw_status": ["code", "message"],
        "kw_field": ["data", "numel"],
        "kw_schedule": [f for f, _ in __import__("kwave._lib", fromlist=["KwSchedule"]).KwSchedule._fields_],
    }
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for s, fields in structs.items():
        lines.append(f'printf("{s} sizeof %zu\\n", sizeof({s}));')
        for f in fields:
            lines.append(f'printf("{s} {f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        s, f, v = line.split()
        res[(s, f)] = int(v)
    return res


def test_ctypes_layout_matches_c_header():
    from kwave import _lib

    c = _c_layout()
    for name, cls in [("kw_input", _lib.KwInput), ("kw_options", _lib.KwOptions), ("kw_output", _lib.KwOutput),
                      ("kw_output_sizes", _lib.KwOutputSizes), ("kw_status", _lib.KwStatus),
                      ("kw_field", _lib.KwField), ("kw_schedule", _lib.KwSchedule)]:
        assert C.sizeof(cls) == c[(name, "sizeof")], name
        for f, _ in cls._fields_:
            assert getattr(cls, f).offset == c[(name, f)], f"{name}.{f}"


def test_output_sizes_query_without_gpu():
    from kwave import _lib
    from helpers import case_3d_het

    inp, record, start, _ = case_3d_het(n=(32, 36, 40), nt=25)
    s, keep = _lib.make_input(inp)
    opt = _lib.make_options(record, start_index=5)
    sz = _lib.output_sizes(s, opt)
    assert sz.num_sensor_points == int(np.asarray(inp["sensor_mask_index"]).size)
    assert sz.num_recorded_steps == 25 - 5 + 1
    assert sz.grid_points == 32 * 36 * 40
    # cuboid corners: 6 x K, sizes from the corners
    inp2 = dict(inp)
    inp2["sensor_mask_type"] = 1
    inp2["sensor_mask_corners"] = np.array([[1, 1, 1, 4, 5, 6], [2, 3, 4, 2, 3, 4]]).T
    s2, keep2 = _lib.make_input(inp2)
    assert _lib.output_sizes(s2, opt).num_sensor_points == 4 * 5 * 6 + 1


def test_invalid_inputs_fail_on_the_host():
    """Validation happens before any device work, so these errors need no GPU."""
    from kwave import _lib
    from helpers import case_2d_p0

    inp, record, start, _ = case_2d_p0()
    bad = dict(inp)
    bad["Nx"] = 11 * 8  # a prime factor above 7
    with pytest.raises(_lib.KwaveError) as e:
        _lib.solve(bad, record)
    assert e.value.code == 5  # KW_ERR_UNSUPPORTED
    bad = dict(inp)
    bad["c0"] = np.ones(17)  # neither a scalar nor a full grid
    with pytest.raises(_lib.KwaveError) as e:
        _lib.solve(bad, record)
    assert e.value.code == 1  # KW_ERR_INVALID_ARGUMENT
    bad = dict(inp)
    bad["sensor_mask_type"] = 1
    bad["sensor_mask_corners"] = np.array([[1, 2, 3, 4, 5]])
    s, keep = _lib.make_input(bad)
    with pytest.raises(_lib.KwaveError):
        _lib.output_sizes(s, _lib.make_options(record))
