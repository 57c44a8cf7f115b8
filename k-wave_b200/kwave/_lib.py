"""ctypes binding of ``include/kwave_b200.h``.

The structures mirror the C declarations field by field.  ``solve()`` takes
the datasets of a k-Wave HDF5 input file as a dict (the names written by
``k-Wave/private/kspaceFirstOrder_saveToDisk.m``) and returns the datasets
of the output file (the names read by ``k-Wave/kspaceFirstOrder3DC.m:569-776``).

There is no fallback: if the shared library is missing, importing this
module raises, and every solve runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("KWAVE_B200_LIB", os.path.join(os.path.dirname(_HERE), "libkwave_b200.so"))

(KW_OK, KW_ERR_INVALID_ARGUMENT, KW_ERR_CUDA, KW_ERR_OUT_OF_MEMORY, KW_ERR_IO, KW_ERR_UNSUPPORTED,
 KW_ERR_INTERNAL) = range(7)
STATUS_NAMES = {0: "KW_OK", 1: "KW_ERR_INVALID_ARGUMENT", 2: "KW_ERR_CUDA", 3: "KW_ERR_OUT_OF_MEMORY",
                4: "KW_ERR_IO", 5: "KW_ERR_UNSUPPORTED", 6: "KW_ERR_INTERNAL"}

c_float_p = C.POINTER(C.c_float)
c_u64_p = C.POINTER(C.c_uint64)


class KwStatus(C.Structure):
    _fields_ = [("code", C.c_int), ("message", C.c_char * 512)]


class KwField(C.Structure):
    _fields_ = [("data", c_float_p), ("numel", C.c_uint64)]


class KwInput(C.Structure):
    _fields_ = [
        ("Nx", C.c_uint64), ("Ny", C.c_uint64), ("Nz", C.c_uint64), ("Nt", C.c_uint64),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
        ("c_ref", C.c_float),
        ("pml_x_size", C.c_uint64), ("pml_y_size", C.c_uint64), ("pml_z_size", C.c_uint64),
        ("pml_x_alpha", C.c_float), ("pml_y_alpha", C.c_float), ("pml_z_alpha", C.c_float),
        ("c0", KwField), ("rho0", KwField),
        ("rho0_sgx", KwField), ("rho0_sgy", KwField), ("rho0_sgz", KwField),
        ("nonlinear_flag", C.c_uint64), ("BonA", KwField),
        ("absorbing_flag", C.c_uint64), ("alpha_coeff", KwField), ("alpha_power", C.c_float),
        ("p0_source_flag", C.c_uint64), ("p0_source_input", c_float_p),
        ("p_source_flag", C.c_uint64), ("p_source_mode", C.c_uint64), ("p_source_many", C.c_uint64),
        ("p_source_index", c_u64_p), ("p_source_index_numel", C.c_uint64),
        ("p_source_input", c_float_p),
        ("ux_source_flag", C.c_uint64), ("uy_source_flag", C.c_uint64), ("uz_source_flag", C.c_uint64),
        ("u_source_mode", C.c_uint64), ("u_source_many", C.c_uint64),
        ("u_source_index", c_u64_p), ("u_source_index_numel", C.c_uint64),
        ("ux_source_input", c_float_p), ("uy_source_input", c_float_p), ("uz_source_input", c_float_p),
        ("sensor_mask_type", C.c_uint64),
        ("sensor_mask_index", c_u64_p), ("sensor_mask_index_numel", C.c_uint64),
        ("sensor_mask_corners", c_u64_p), ("sensor_mask_corners_numel", C.c_uint64),
        ("transducer_source_flag", C.c_uint64), ("transducer_source_input", c_float_p),
        ("transducer_source_input_numel", C.c_uint64), ("delay_mask", c_u64_p),
        ("transducer_source_apodization", c_float_p),
        ("axisymmetric_flag", C.c_uint64),
        ("sensor_interp_index", c_u64_p), ("sensor_interp_weight", c_float_p),
        ("sensor_interp_numel", C.c_uint64),
    ]


class KwOptions(C.Structure):
    _fields_ = [
        ("p_raw", C.c_int), ("p_max", C.c_int), ("p_min", C.c_int), ("p_rms", C.c_int),
        ("p_max_all", C.c_int), ("p_min_all", C.c_int), ("p_final", C.c_int),
        ("u_raw", C.c_int), ("u_max", C.c_int), ("u_min", C.c_int), ("u_rms", C.c_int),
        ("u_max_all", C.c_int), ("u_min_all", C.c_int), ("u_final", C.c_int),
        ("u_non_staggered_raw", C.c_int),
        ("start_index", C.c_uint64), ("device", C.c_int), ("verbose", C.c_int),
    ]


OUTPUT_FIELDS = [
    "p", "p_max", "p_min", "p_rms", "p_max_all", "p_min_all", "p_final",
    "ux", "uy", "uz", "ux_max", "uy_max", "uz_max", "ux_min", "uy_min", "uz_min",
    "ux_rms", "uy_rms", "uz_rms", "ux_max_all", "uy_max_all", "uz_max_all",
    "ux_min_all", "uy_min_all", "uz_min_all", "ux_final", "uy_final", "uz_final",
    "ux_non_staggered", "uy_non_staggered", "uz_non_staggered",
]


class KwOutput(C.Structure):
    _fields_ = [(n, c_float_p) for n in OUTPUT_FIELDS]


class KwSchedule(C.Structure):
    _fields_ = [("slab_planes", C.c_int), ("streams", C.c_int), ("row_lines", C.c_int), ("col_lines", C.c_int),
                ("radix_plan", C.c_int), ("candidates", C.c_int), ("ms_per_step", C.c_float),
                ("ms_default", C.c_float)]


class KwOutputSizes(C.Structure):
    _fields_ = [("num_sensor_points", C.c_uint64), ("num_recorded_steps", C.c_uint64),
                ("grid_points", C.c_uint64), ("device_bytes", C.c_uint64)]


EXPORTED = [
    "kw_version", "kw_output_sizes_query", "kw_solve", "kw_run_file", "kw_run_file_checkpointed", "kw_cli_main",
    "kw_session_create", "kw_session_advance", "kw_session_elapsed_ms", "kw_session_sync",
    "kw_session_steps_done", "kw_session_read", "kw_session_stream", "kw_session_launches_per_step",
    "kw_session_destroy", "kw_session_query", "kw_stream_priority_range", "kw_session_set_priority",
    "kw_session_save", "kw_session_restore",
    "kw_tune", "kw_wisdom_import", "kw_wisdom_export", "kw_wisdom_forget", "kw_session_schedule",
    "kw_batch_create", "kw_batch_advance", "kw_batch_elapsed_ms", "kw_batch_sync", "kw_batch_graph_launches",
    "kw_batch_destroy",
    "kw_kspace_gradient_noalloc",
    "kw_fft3d_create", "kw_fft3d_exec", "kw_fft3d_check", "kw_fft3d_destroy",
]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"kwave_b200 shared library not found at {LIB_PATH}; "
                          "build it with `python k-wave_b200/build.py`")
    lib = C.CDLL(LIB_PATH)
    lib.kw_version.restype = C.c_char_p
    lib.kw_output_sizes_query.argtypes = [C.POINTER(KwInput), C.POINTER(KwOptions),
                                          C.POINTER(KwOutputSizes), C.POINTER(KwStatus)]
    lib.kw_solve.argtypes = [C.POINTER(KwInput), C.POINTER(KwOptions), C.POINTER(KwOutput),
                             C.POINTER(KwStatus)]
    lib.kw_run_file.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(KwOptions), C.POINTER(KwStatus)]
    lib.kw_cli_main.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
    lib.kw_run_file_checkpointed.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(KwOptions), C.c_char_p, C.c_uint64,
                                             C.c_double, C.POINTER(KwStatus)]
    lib.kw_session_create.argtypes = [C.POINTER(KwInput), C.POINTER(KwOptions), C.POINTER(C.c_void_p),
                                      C.POINTER(KwStatus)]
    lib.kw_session_advance.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(KwStatus)]
    lib.kw_session_elapsed_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(KwStatus)]
    lib.kw_session_sync.argtypes = [C.c_void_p, C.POINTER(KwStatus)]
    lib.kw_session_steps_done.argtypes = [C.c_void_p]
    lib.kw_session_steps_done.restype = C.c_uint64
    lib.kw_session_query.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(KwStatus)]
    lib.kw_stream_priority_range.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.kw_session_set_priority.argtypes = [C.c_void_p, C.c_int, C.POINTER(KwStatus)]
    lib.kw_session_save.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(KwStatus)]
    lib.kw_session_restore.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(KwStatus)]
    lib.kw_session_read.argtypes = [C.c_void_p, C.POINTER(KwOutput), C.POINTER(KwStatus)]
    lib.kw_session_stream.argtypes = [C.c_void_p]
    lib.kw_session_stream.restype = C.c_void_p
    lib.kw_session_launches_per_step.argtypes = [C.c_void_p]
    lib.kw_session_launches_per_step.restype = C.c_uint64
    lib.kw_session_destroy.argtypes = [C.c_void_p]
    lib.kw_tune.argtypes = [C.POINTER(KwInput), C.POINTER(KwOptions), C.POINTER(KwSchedule), C.POINTER(KwStatus)]
    lib.kw_wisdom_import.argtypes = [C.c_char_p, C.POINTER(KwStatus)]
    lib.kw_wisdom_export.argtypes = [C.c_char_p, C.POINTER(KwStatus)]
    lib.kw_wisdom_forget.argtypes = []
    lib.kw_wisdom_forget.restype = None
    lib.kw_session_schedule.argtypes = [C.c_void_p, C.POINTER(KwSchedule)]
    lib.kw_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p), C.POINTER(KwStatus)]
    lib.kw_batch_advance.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(KwStatus)]
    lib.kw_batch_elapsed_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(KwStatus)]
    lib.kw_batch_sync.argtypes = [C.c_void_p, C.POINTER(KwStatus)]
    lib.kw_batch_graph_launches.argtypes = [C.c_void_p]
    lib.kw_batch_graph_launches.restype = C.c_uint64
    lib.kw_batch_destroy.argtypes = [C.c_void_p]
    lib.kw_kspace_gradient_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                               C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p,
                                               C.POINTER(KwStatus)]
    lib.kw_fft3d_create.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(C.c_void_p), C.POINTER(KwStatus)]
    lib.kw_fft3d_exec.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(KwStatus)]
    lib.kw_fft3d_check.argtypes = [C.c_void_p, C.POINTER(KwStatus)]
    lib.kw_fft3d_destroy.argtypes = [C.c_void_p]
    lib.kw_fft3d_destroy.restype = None
    return lib


lib = _load()


class KwaveError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def _check(code, st):
    if code != KW_OK:
        raise KwaveError(code, st.message.decode(errors="replace"))


# ---------------------------------------------------------------------------
# dict <-> struct
# ---------------------------------------------------------------------------
RECORD_TO_FLAG = {
    "p": "p_raw", "p_max": "p_max", "p_min": "p_min", "p_rms": "p_rms", "p_max_all": "p_max_all",
    "p_min_all": "p_min_all", "p_final": "p_final", "u": "u_raw", "u_max": "u_max", "u_min": "u_min",
    "u_rms": "u_rms", "u_max_all": "u_max_all", "u_min_all": "u_min_all", "u_final": "u_final",
    "u_non_staggered": "u_non_staggered_raw",
}


def make_options(record=("p",), start_index=1, device=-1, verbose=0):
    o = KwOptions()
    for r in record:
        setattr(o, RECORD_TO_FLAG[r], 1)
    o.start_index = int(start_index)
    o.device = int(device)
    o.verbose = int(verbose)
    return o


class _Keep:
    """Holds the numpy arrays a KwInput points into."""

    def __init__(self):
        self.arrays = []

    def f32(self, v):
        a = np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(-1, order="F"))
        self.arrays.append(a)
        return a

    def u64(self, v):
        a = np.ascontiguousarray(np.asarray(v, dtype=np.uint64).reshape(-1, order="F"))
        self.arrays.append(a)
        return a


def _fptr(a):
    return a.ctypes.data_as(c_float_p)


def _uptr(a):
    return a.ctypes.data_as(c_u64_p)


def make_input(inp: dict):
    """Build a KwInput from HDF5-file-level datasets.

    Grid arrays are accepted in MATLAB axis order (shape (Nx, Ny[, Nz])) and
    flattened x-fastest; signal matrices are (rows, Nt_src) as in MATLAB."""
    keep = _Keep()
    s = KwInput()
    for k in ("Nx", "Ny", "Nz", "Nt"):
        setattr(s, k, int(inp[k]))
    for k in ("dx", "dy", "dz", "dt", "c_ref"):
        setattr(s, k, float(inp.get(k, 0.0)))
    for a in "xyz":
        setattr(s, f"pml_{a}_size", int(inp.get(f"pml_{a}_size", 0)))
        setattr(s, f"pml_{a}_alpha", float(inp.get(f"pml_{a}_alpha", 0.0)))

    def fld(name):
        if name not in inp or inp[name] is None:
            return KwField()
        a = keep.f32(inp[name])
        return KwField(_fptr(a), a.size)

    for name in ("c0", "rho0", "rho0_sgx", "rho0_sgy", "rho0_sgz", "BonA", "alpha_coeff"):
        setattr(s, name, fld(name))
    s.nonlinear_flag = int(inp.get("nonlinear_flag", 0))
    s.absorbing_flag = int(inp.get("absorbing_flag", 0))
    s.alpha_power = float(inp.get("alpha_power", 0.0))
    s.p0_source_flag = int(inp.get("p0_source_flag", 0))
    if s.p0_source_flag:
        s.p0_source_input = _fptr(keep.f32(inp["p0_source_input"]))
    s.p_source_flag = int(inp.get("p_source_flag", 0))
    if s.p_source_flag:
        s.p_source_mode = int(inp["p_source_mode"])
        s.p_source_many = int(inp.get("p_source_many", 0))
        idx = keep.u64(inp["p_source_index"])
        s.p_source_index = _uptr(idx)
        s.p_source_index_numel = idx.size
        sig = np.asarray(inp["p_source_input"], dtype=np.float32)
        sig = sig.reshape(-1, sig.shape[-1]) if sig.ndim > 1 else sig.reshape(1, -1)
        # [rows, t] column-major == [t][rows] row-fastest
        s.p_source_input = _fptr(keep.f32(sig))
    u_any = False
    for a in "xyz":
        fl = int(inp.get(f"u{a}_source_flag", 0))
        setattr(s, f"u{a}_source_flag", fl)
        if fl:
            u_any = True
            sig = np.asarray(inp[f"u{a}_source_input"], dtype=np.float32)
            sig = sig.reshape(-1, sig.shape[-1]) if sig.ndim > 1 else sig.reshape(1, -1)
            setattr(s, f"u{a}_source_input", _fptr(keep.f32(sig)))
    s.axisymmetric_flag = int(inp.get("axisymmetric_flag", 0))
    s.transducer_source_flag = int(inp.get("transducer_source_flag", 0))
    if u_any or s.transducer_source_flag:
        s.u_source_mode = int(inp.get("u_source_mode", 0))
        s.u_source_many = int(inp.get("u_source_many", 0))
        idx = keep.u64(inp["u_source_index"])
        s.u_source_index = _uptr(idx)
        s.u_source_index_numel = idx.size
    if s.transducer_source_flag:
        sig = keep.f32(inp["transducer_source_input"])
        s.transducer_source_input = _fptr(sig)
        s.transducer_source_input_numel = sig.size
        s.delay_mask = _uptr(keep.u64(inp["delay_mask"]))
        if inp.get("transducer_source_apodization") is not None:
            s.transducer_source_apodization = _fptr(keep.f32(inp["transducer_source_apodization"]))
    s.sensor_mask_type = int(inp.get("sensor_mask_type", 0))
    if inp.get("sensor_interp_index") is not None:
        # (points, Nd + 1) arrays, flattened point-major (C order)
        vi = np.ascontiguousarray(np.asarray(inp["sensor_interp_index"], dtype=np.uint64).reshape(-1))
        vw = np.ascontiguousarray(np.asarray(inp["sensor_interp_weight"], dtype=np.float32).reshape(-1))
        keep.arrays += [vi, vw]
        if vi.size != vw.size:
            raise ValueError("sensor_interp_index and sensor_interp_weight differ in size")
        s.sensor_interp_index = _uptr(vi)
        s.sensor_interp_weight = _fptr(vw)
        s.sensor_interp_numel = vi.size
    elif s.sensor_mask_type == 0:
        idx = keep.u64(inp["sensor_mask_index"])
        s.sensor_mask_index = _uptr(idx)
        s.sensor_mask_index_numel = idx.size
    else:
        cor = keep.u64(inp["sensor_mask_corners"])  # (6, K) column-major: one cuboid per 6 values
        s.sensor_mask_corners = _uptr(cor)
        s.sensor_mask_corners_numel = cor.size
    return s, keep


def output_sizes(inp_struct, opt):
    st = KwStatus()
    sz = KwOutputSizes()
    _check(lib.kw_output_sizes_query(C.byref(inp_struct), C.byref(opt), C.byref(sz), C.byref(st)), st)
    return sz


def alloc_outputs(inp: dict, record, sizes):
    """Host buffers (numpy) for the requested outputs and the KwOutput struct."""
    dim = 2 if int(inp["Nz"]) == 1 else 3
    ns, nr, ng = sizes.num_sensor_points, sizes.num_recorded_steps, sizes.grid_points
    comps = "xyz"[:dim]
    bufs = {}
    rec = set(record)
    if "p" in rec:
        bufs["p"] = np.zeros((nr, ns), np.float32)
    for k in ("p_max", "p_min", "p_rms"):
        if k in rec:
            bufs[k] = np.zeros(ns, np.float32)
    for k in ("p_max_all", "p_min_all", "p_final"):
        if k in rec:
            bufs[k] = np.zeros(ng, np.float32)
    for c in comps:
        if "u" in rec:
            bufs["u" + c] = np.zeros((nr, ns), np.float32)
        for k in ("max", "min", "rms"):
            if "u_" + k in rec:
                bufs[f"u{c}_{k}"] = np.zeros(ns, np.float32)
        for k in ("max_all", "min_all", "final"):
            if "u_" + k in rec:
                bufs[f"u{c}_{k}"] = np.zeros(ng, np.float32)
        if "u_non_staggered" in rec:
            bufs[f"u{c}_non_staggered"] = np.zeros((nr, ns), np.float32)
    out = KwOutput()
    for k, v in bufs.items():
        setattr(out, k, _fptr(v))
    return out, bufs


def to_matlab_layout(bufs: dict, inp: dict):
    """Convert output buffers to the reference's array shapes: time series
    (Ns, Nt_rec); per-point (Ns,); grid outputs (Nx, Ny[, Nz])."""
    dim = 2 if int(inp["Nz"]) == 1 else 3
    shape = (int(inp["Nx"]), int(inp["Ny"])) + ((int(inp["Nz"]),) if dim == 3 else ())
    res = {}
    for k, v in bufs.items():
        if v.ndim == 2:
            res[k] = v.T
        elif k.endswith("_all") or k.endswith("_final"):
            res[k] = v.reshape(shape, order="F")
        else:
            res[k] = v
    return res


def solve(inp: dict, record=("p",), start_index=1, device=-1):
    """kw_solve(): one simulation, host buffers in and out."""
    s, keep = make_input(inp)
    opt = make_options(record, start_index, device)
    sizes = output_sizes(s, opt)
    out, bufs = alloc_outputs(inp, record, sizes)
    st = KwStatus()
    _check(lib.kw_solve(C.byref(s), C.byref(opt), C.byref(out), C.byref(st)), st)
    del keep
    return to_matlab_layout(bufs, inp)


def run_file(input_path, output_path, record=("p",), start_index=1, device=-1, verbose=0, checkpoint=None,
             checkpoint_timesteps=0, checkpoint_interval=0.0):
    """kw_run_file(): read a k-Wave HDF5 input file, run it, write the output
    file (what kspaceFirstOrder3DC.m:560-567 does through the binary).  With
    `checkpoint`, the state is saved there every `checkpoint_timesteps` steps
    and / or `checkpoint_interval` seconds and resumed from if it exists."""
    opt = make_options(record, start_index, device, verbose)
    st = KwStatus()
    if checkpoint is None:
        _check(lib.kw_run_file(os.fsencode(input_path), os.fsencode(output_path), C.byref(opt), C.byref(st)), st)
    else:
        _check(lib.kw_run_file_checkpointed(os.fsencode(input_path), os.fsencode(output_path), C.byref(opt),
                                            os.fsencode(checkpoint), int(checkpoint_timesteps),
                                            float(checkpoint_interval), C.byref(st)), st)


def cli_main(argv):
    """kw_cli_main(): the command line of the solver binary, in process."""
    args = [os.fsencode(a) for a in argv]
    arr = (C.c_char_p * len(args))(*args)
    return lib.kw_cli_main(len(args), arr)


class Session:
    """A resident simulation advanced in steps (kw_session_*)."""

    def __init__(self, inp: dict, record=("p",), start_index=1, device=-1):
        self.inp = inp
        self.record = tuple(record)
        self._s, self._keep = make_input(inp)
        self._opt = make_options(record, start_index, device)
        self.sizes = output_sizes(self._s, self._opt)
        h = C.c_void_p()
        st = KwStatus()
        _check(lib.kw_session_create(C.byref(self._s), C.byref(self._opt), C.byref(h), C.byref(st)), st)
        self._h = h

    def advance(self, n):
        st = KwStatus()
        _check(lib.kw_session_advance(self._h, C.c_uint64(int(n)), C.byref(st)), st)

    def elapsed_ms(self):
        st = KwStatus()
        ms = C.c_float()
        _check(lib.kw_session_elapsed_ms(self._h, C.byref(ms), C.byref(st)), st)
        return ms.value

    def sync(self):
        st = KwStatus()
        _check(lib.kw_session_sync(self._h, C.byref(st)), st)

    @property
    def steps_done(self):
        return int(lib.kw_session_steps_done(self._h))

    def save(self, path):
        """Write a checkpoint of the state between two steps (waits for queued work)."""
        st = KwStatus()
        _check(lib.kw_session_save(self._h, os.fsencode(path), C.byref(st)), st)

    def restore(self, path):
        """Continue from a checkpoint (this session must be fresh, same input and options)."""
        st = KwStatus()
        _check(lib.kw_session_restore(self._h, os.fsencode(path), C.byref(st)), st)

    def set_priority(self, priority):
        """CUDA stream priority of the session's work (lower runs first)."""
        st = KwStatus()
        _check(lib.kw_session_set_priority(self._h, int(priority), C.byref(st)), st)

    def in_flight(self):
        """How many advance() calls still have steps running on the device."""
        st = KwStatus()
        n = C.c_uint64(0)
        _check(lib.kw_session_query(self._h, C.byref(n), C.byref(st)), st)
        return int(n.value)

    @property
    def stream(self):
        return lib.kw_session_stream(self._h)

    @property
    def launches_per_step(self):
        return int(lib.kw_session_launches_per_step(self._h))

    @property
    def schedule(self):
        """The launch schedule the session runs with (kw_session_schedule)."""
        sc = KwSchedule()
        code = lib.kw_session_schedule(self._h, C.byref(sc))
        if code != KW_OK:
            raise KwaveError(code, "kw_session_schedule")
        return _schedule_dict(sc)

    def read(self):
        out, bufs = alloc_outputs(self.inp, self.record, self.sizes)
        st = KwStatus()
        _check(lib.kw_session_read(self._h, C.byref(out), C.byref(st)), st)
        return to_matlab_layout(bufs, self.inp)

    def close(self):
        if getattr(self, "_h", None):
            lib.kw_session_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Batch:
    """Sessions advanced together, one CUDA graph launch per time step for
    all of them (kw_batch_*).  The sessions stay owned by the caller."""

    def __init__(self, sessions):
        self.sessions = list(sessions)
        arr = (C.c_void_p * len(self.sessions))(*[s._h.value for s in self.sessions])
        h = C.c_void_p()
        st = KwStatus()
        _check(lib.kw_batch_create(arr, len(self.sessions), C.byref(h), C.byref(st)), st)
        self._h = h

    def advance(self, n):
        if any(not getattr(s, "_h", None) for s in self.sessions):
            raise KwaveError(KW_ERR_INVALID_ARGUMENT, "a session of the batch was closed")
        st = KwStatus()
        _check(lib.kw_batch_advance(self._h, C.c_uint64(int(n)), C.byref(st)), st)

    def elapsed_ms(self):
        st = KwStatus()
        ms = C.c_float()
        _check(lib.kw_batch_elapsed_ms(self._h, C.byref(ms), C.byref(st)), st)
        return ms.value

    def sync(self):
        st = KwStatus()
        _check(lib.kw_batch_sync(self._h, C.byref(st)), st)

    @property
    def graph_launches(self):
        return int(lib.kw_batch_graph_launches(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib.kw_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _schedule_dict(sc):
    return {"slab_planes": sc.slab_planes, "streams": sc.streams, "row_lines": sc.row_lines,
            "col_lines": sc.col_lines, "radix_plan": sc.radix_plan, "candidates": sc.candidates,
            "ms_per_step": sc.ms_per_step, "ms_default": sc.ms_default}


def tune(inp: dict, record=("p",), start_index=1, device=-1):
    """kw_tune(): time the launch schedules of this simulation's step on a
    scratch copy and remember the fastest for its grid and step class.
    Returns the chosen schedule with the measured ms per step."""
    s, keep = make_input(inp)
    opt = make_options(record, start_index, device)
    sc = KwSchedule()
    st = KwStatus()
    _check(lib.kw_tune(C.byref(s), C.byref(opt), C.byref(sc), C.byref(st)), st)
    del keep
    return _schedule_dict(sc)


def wisdom_import(path):
    st = KwStatus()
    _check(lib.kw_wisdom_import(os.fsencode(path), C.byref(st)), st)


def wisdom_export(path):
    st = KwStatus()
    _check(lib.kw_wisdom_export(os.fsencode(path), C.byref(st)), st)


def wisdom_forget():
    lib.kw_wisdom_forget()


def stream_priority_range():
    """(least, greatest) CUDA stream priorities of the current device."""
    lo, hi = C.c_int(0), C.c_int(0)
    lib.kw_stream_priority_range(C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def kspace_gradient_noalloc(d_f, d_gx, d_gy, nx, ny, dx, dy, c_ref, dt, stream=None):
    """kw_kspace_gradient_noalloc(): device pointers (ints) in, nothing
    allocated; the work is only enqueued on `stream` (a cudaStream_t handle)."""
    st = KwStatus()
    _check(lib.kw_kspace_gradient_noalloc(d_f, d_gx, d_gy, int(nx), int(ny), float(dx), float(dy), float(c_ref),
                                          float(dt), stream, C.byref(st)), st)


class Fft3d:
    """kw_fft3d_*: the solver's own FFT passes as a plain real-to-complex
    transform of an nx x ny x nz grid (nz = 1: 2D), on device buffers given
    as integer pointers.  Spectrum layout [nz][ny][nxp] complex64 with
    nxp = nx // 2 + 1 rounded up to even; the inverse is unnormalised."""

    def __init__(self, nx, ny, nz=1):
        self.shape = (int(nx), int(ny), int(nz))
        self.nxp = (int(nx) // 2 + 2) // 2 * 2
        h = C.c_void_p()
        st = KwStatus()
        _check(lib.kw_fft3d_create(int(nx), int(ny), int(nz), C.byref(h), C.byref(st)), st)
        self._h = h

    def exec(self, d_real, d_spec, inverse=False, passes=7, stream=None):
        st = KwStatus()
        _check(lib.kw_fft3d_exec(self._h, int(bool(inverse)), int(passes), d_real, d_spec, stream, C.byref(st)), st)

    def check(self):
        st = KwStatus()
        _check(lib.kw_fft3d_check(self._h, C.byref(st)), st)

    def close(self):
        if getattr(self, "_h", None):
            lib.kw_fft3d_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def version():
    return lib.kw_version().decode()
