"""The HDF5 file boundary without a GPU: the C reader/writer inside
libkwave_b200.so and the independent Python one in kwave.h5io are checked
against published known answers, a file written by MATLAB's HDF5 library,
and each other; the input-file reader of kw_run_file and the command line
are checked up to the point where the solver would need a device."""
import ctypes as C
import os
import struct
import subprocess

import numpy as np
import pytest

from helpers import case_2d_p0, case_3d_het

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "k-wave_b200", "kspaceFirstOrder-B200")
# a MATLAB 7.3 (HDF5) file shipped with scipy's test data in this image
MATLAB_73 = None
try:
    import scipy.io.matlab as _sm

    MATLAB_73 = os.path.join(os.path.dirname(_sm.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
except ImportError:
    pass
# a chunked + deflated MATLAB 7.3 file of the reference's example data, read
# when KWAVE_B200_REFERENCE_TREE names a checkout of the reference (k-Wave/...)
_REF_TREE = os.environ.get("KWAVE_B200_REFERENCE_TREE")
REF_EXAMPLE = os.path.join(_REF_TREE, "k-Wave", "examples", "EXAMPLE_shepp_logan.mat") if _REF_TREE else None


def _lib():
    from kwave import _lib

    L = _lib.lib
    L.kwb_h5_lookup3.restype = C.c_uint32
    L.kwb_h5_lookup3.argtypes = [C.c_char_p, C.c_size_t, C.c_uint32]
    L.kwb_h5_read.restype = C.c_int64
    L.kwb_h5_read.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_int),
                              C.c_char_p, C.c_int]
    L.kwb_h5_read_attribute.restype = C.c_int64
    L.kwb_h5_read_attribute.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
    L.kwb_h5_write.restype = C.c_int
    return L


def c_read(path, name, cap=1 << 22):
    L = _lib()
    out = np.zeros(cap)
    dims = np.zeros(8, np.uint64)
    rank = C.c_int()
    err = C.create_string_buffer(512)
    n = L.kwb_h5_read(os.fsencode(path), name.encode(), out.ctypes.data, cap, dims.ctypes.data, C.byref(rank), err,
                      512)
    if n < 0:
        raise ValueError(err.value.decode())
    return out[:n].reshape(tuple(int(d) for d in dims[:rank.value]))


def c_attr(path, obj, name):
    buf = C.create_string_buffer(512)
    assert _lib().kwb_h5_read_attribute(os.fsencode(path), obj.encode(), name.encode(), buf, 512) == 0
    return buf.value.decode()


def c_write(path, items):
    """items: list of (path, numpy array) stored with the array's C shape."""
    L = _lib()
    n = len(items)
    code = {np.dtype(np.float32): 0, np.dtype(np.float64): 1, np.dtype(np.uint64): 2}
    arrays = [np.ascontiguousarray(a) for _, a in items]
    dims = [np.asarray(a.shape, np.uint64) for a in arrays]
    paths = (C.c_char_p * n)(*[p.encode() for p, _ in items])
    types = (C.c_int * n)(*[code[a.dtype] for a in arrays])
    dptr = (C.c_void_p * n)(*[d.ctypes.data for d in dims])
    ranks = (C.c_int * n)(*[a.ndim for a in arrays])
    data = (C.c_void_p * n)(*[a.ctypes.data for a in arrays])
    err = C.create_string_buffer(512)
    rc = L.kwb_h5_write(os.fsencode(path), n, paths, types, dptr, ranks, data, err, 512)
    assert rc == 0, err.value


def verify_checksums(path):
    """Every version-2 superblock / object header of the file carries a
    valid lookup3 checksum (what libhdf5 checks when it opens the file)."""
    from kwave import h5io

    raw = open(path, "rb").read()
    assert raw[:8] == h5io.SIG and raw[8] == 2
    assert struct.unpack("<I", raw[44:48])[0] == h5io.lookup3(raw[:44])
    n = 0
    pos = raw.find(b"OHDR")
    while pos >= 0:
        flags = raw[pos + 5]
        nb = 1 << (flags & 3)
        size = int.from_bytes(raw[pos + 6:pos + 6 + nb], "little")
        end = pos + 6 + nb + size
        assert struct.unpack("<I", raw[end:end + 4])[0] == h5io.lookup3(raw[pos:end]), f"OHDR at {pos}"
        n += 1
        pos = raw.find(b"OHDR", end + 4)
    return n


# ---------------------------------------------------------------------------
def test_lookup3_known_answers():
    """Known answers published with lookup3.c (driver5)."""
    from kwave import h5io

    L = _lib()
    s = b"Four score and seven years ago"
    cases = [(b"", 0, 0xDEADBEEF), (b"", 0xDEADBEEF, 0xBD5B7DDE), (s, 0, 0x17770551), (s, 1, 0xCD628161)]
    for data, init, want in cases:
        assert L.kwb_h5_lookup3(data, len(data), init) == want
        assert h5io.lookup3(data, init) == want


@pytest.mark.skipif(MATLAB_73 is None or not os.path.exists(MATLAB_73), reason="MATLAB 7.3 fixture absent")
def test_matlab_written_file():
    """Superblock behind a 512-byte user block, v1 object headers, symbol
    table group, layout v2: MATLAB stores testdouble = 0:pi/4:2*pi."""
    from kwave import h5io

    want = np.pi / 4 * np.arange(9)
    np.testing.assert_allclose(h5io.read(MATLAB_73, "/testdouble").reshape(-1), want, rtol=0, atol=1e-15)
    np.testing.assert_allclose(c_read(MATLAB_73, "/testdouble").reshape(-1), want, rtol=0, atol=1e-15)
    assert c_read(MATLAB_73, "/testdouble").shape == (9, 1)
    assert c_attr(MATLAB_73, "/testdouble", "MATLAB_class") == "double"
    with h5io.File(MATLAB_73) as f:
        assert f.attrs("/testdouble")["MATLAB_class"] == "double"


@pytest.mark.skipif(not (REF_EXAMPLE and os.path.exists(REF_EXAMPLE)), reason="KWAVE_B200_REFERENCE_TREE unset or its example data absent")
def test_chunked_deflated_matlab_file():
    """Chunked (B-tree v1) + deflate: both readers agree bit for bit on the
    modified Shepp-Logan phantom, whose intensities are 0, .1, .2, .3, .4, 1."""
    from kwave import h5io

    a = h5io.read(REF_EXAMPLE, "/shepp_logan")
    b = c_read(REF_EXAMPLE, "/shepp_logan")
    assert a.shape == b.shape == (472, 472)
    assert np.array_equal(a, b)
    np.testing.assert_allclose(np.unique(np.round(a, 6)), [0, 0.1, 0.2, 0.3, 0.4, 1.0])


def test_python_writer_c_reader(tmp_path):
    from kwave import h5io

    rng = np.random.default_rng(3)
    f = tmp_path / "py.h5"
    w = h5io.Writer()
    items = {
        "/a": rng.standard_normal((3, 4, 5)).astype(np.float32),
        "/b": np.arange(7, dtype=np.uint64)[None, None, :],
        "/g/h/c": rng.standard_normal((2, 6)),
        "/empty": np.zeros((1, 0, 1), np.float32),
    }
    for k, v in items.items():
        w.dataset(k, v, {"data_type": "float", "domain_type": "real"})
    w.attribute("file_type", "input")
    w.write(f)
    assert verify_checksums(f) == 7  # root, g, g/h, 4 datasets
    for k, v in items.items():
        got = c_read(f, k)
        assert got.shape == v.shape
        assert np.array_equal(got, v.astype(np.float64))
        assert np.array_equal(h5io.read(f, k), v)
    assert c_attr(f, "/", "file_type") == "input"
    assert c_attr(f, "/a", "domain_type") == "real"
    with pytest.raises(ValueError, match="no object"):
        c_read(f, "/nope")


def test_c_writer_python_reader(tmp_path):
    from kwave import h5io

    rng = np.random.default_rng(4)
    f = tmp_path / "c.h5"
    items = [("/p", rng.standard_normal((1, 17, 5)).astype(np.float32)),
             ("/Nx", np.array([[[64]]], np.uint64)),
             ("/p_max/1", rng.standard_normal((2, 3, 4)).astype(np.float32)),
             ("/p_max/2", rng.standard_normal((1, 3, 1)).astype(np.float32)),
             ("/d", rng.standard_normal(11))]
    c_write(f, items)
    assert verify_checksums(f) == 7
    for k, v in items:
        got = h5io.read(f, k)
        assert got.dtype == v.dtype and got.shape == v.shape
        assert np.array_equal(got, v)
    with h5io.File(f) as F:
        assert F.attrs("/")["file_type"] == "output"
        assert F.attrs("/p")["data_type"] == "float"
        assert F.attrs("/Nx")["data_type"] == "long"


def test_input_file_layout(tmp_path):
    """write_input_file stores MATLAB arrays x-fastest with reversed dims,
    floats as single and indices as uint64, and drops z variables in 2D
    (kspaceFirstOrder_saveToDisk.m:419-427)."""
    from kwave import h5io

    inp, record, start, meta = case_2d_p0(n=(20, 12), nt=10)
    f = tmp_path / "in2d.h5"
    h5io.write_input_file(f, inp)
    with h5io.File(f) as F:
        names = F.children(F.root)
        assert "dz" not in names and "rho0_sgz" not in names and "pml_z_alpha" not in names
        assert "Nz" in names and "pml_z_size" in names
        assert F.attrs("/")["file_type"] == "input"
        assert F.attrs("/")["minor_version"] == "2"
        p0 = F.read("/p0_source_input")
        assert p0.dtype == np.float32 and p0.shape == (1, 12, 20)
        np.testing.assert_array_equal(p0[0].T, np.asarray(inp["p0_source_input"], np.float32))
        idx = F.read("/sensor_mask_index")
        assert idx.dtype == np.uint64
        np.testing.assert_array_equal(idx.reshape(-1), np.asarray(inp["sensor_mask_index"]).reshape(-1))
    assert h5io.read_matlab(f, "/Nx").reshape(-1)[0] == 20


def _run_file_status(inp_path, out_path, record=("p",)):
    from kwave import _lib

    try:
        _lib.run_file(inp_path, out_path, record)
    except _lib.KwaveError as e:
        return e.code, str(e)
    return 0, ""


def test_run_file_reads_input_up_to_the_device(tmp_path):
    """With no GPU, kw_run_file gets through the whole input file and the
    output-size query, and stops with KW_ERR_CUDA when it needs a device."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU file test covers this")
    from kwave import _lib, h5io

    inp, record, start, meta = case_3d_het(n=(16, 18, 20), nt=8, record=("p", "p_max"))
    f = tmp_path / "in3d.h5"
    h5io.write_input_file(f, inp)
    code, msg = _run_file_status(f, tmp_path / "out.h5", record)
    assert code == _lib.KW_ERR_CUDA, msg
    assert not (tmp_path / "out.h5").exists()


def test_run_file_rejects_bad_inputs(tmp_path):
    from kwave import _lib, h5io

    inp, record, start, meta = case_2d_p0(n=(20, 12), nt=10)
    code, msg = _run_file_status(tmp_path / "absent.h5", tmp_path / "o.h5")
    assert code == _lib.KW_ERR_IO and "absent.h5" in msg

    bad = dict(inp, elastic_flag=1)
    h5io.write_input_file(tmp_path / "el.h5", bad)
    code, msg = _run_file_status(tmp_path / "el.h5", tmp_path / "o.h5")
    assert code == _lib.KW_ERR_UNSUPPORTED and "elastic_flag" in msg

    no_c0 = {k: v for k, v in inp.items() if k != "c0"}
    h5io.write_input_file(tmp_path / "noc0.h5", no_c0)
    code, msg = _run_file_status(tmp_path / "noc0.h5", tmp_path / "o.h5")
    assert code == _lib.KW_ERR_IO and "/c0" in msg

    w = h5io.Writer()
    w.dataset("/Nx", np.array([[[4]]], np.uint64))
    w.attribute("file_type", "output")
    w.write(tmp_path / "out_as_in.h5")
    code, msg = _run_file_status(tmp_path / "out_as_in.h5", tmp_path / "o.h5")
    assert code == _lib.KW_ERR_IO and "not an input file" in msg

    (tmp_path / "junk.h5").write_bytes(b"not hdf5 at all" * 10)
    code, msg = _run_file_status(tmp_path / "junk.h5", tmp_path / "o.h5")
    assert code == _lib.KW_ERR_IO


def test_command_line(tmp_path):
    """Exit codes of the binary's command line: 0 help, 2 usage, 1 failure."""
    from kwave import _lib

    assert os.path.exists(BIN), "build the solver binary first"
    run = lambda *a: subprocess.run([BIN, *a], capture_output=True, text=True, timeout=60)
    r = run("--help")
    assert r.returncode == 0 and "usage" in r.stderr
    assert run().returncode == 2
    assert run("-i", "x.h5").returncode == 2
    assert run("-i", "x.h5", "-o", "y.h5", "--bogus").returncode == 2
    assert run("-i", "x.h5", "-o").returncode == 2
    r = run("-i", str(tmp_path / "missing.h5"), "-o", str(tmp_path / "o.h5"), "--p_max", "-t", "8")
    assert r.returncode == 1 and "missing.h5" in r.stderr
    assert run("-i", "x.h5", "-o", "y.h5", "--checkpoint_file", "c.h5").returncode == 2  # needs an interval
    assert _lib.cli_main(["prog", "--help"]) == 0
    assert _lib.cli_main(["prog", "-i"]) == 2
