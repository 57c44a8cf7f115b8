"""Host-side mirror of ``kspaceFirstOrder2D`` / ``kspaceFirstOrder3D`` and of
their C/G-suffixed drop-in wrappers.

``kspace_first_order(kgrid, medium, source, sensor, **options)`` does what
the reference does on the MATLAB side of the file boundary -- input checking,
p0 smoothing, density on the staggered grids, reference sound speed, source
scaling, sensor index lists (``kspaceFirstOrder_inputChecking.m``,
``kspaceFirstOrder3D.m:583-605``, ``kspaceFirstOrder_scaleSourceTerms.m``,
``kspaceFirstOrder3DC.m:425-525``) -- then runs the time loop on the GPU
through the C ABI (``kw_solve``) and applies the reference's
post-processing (intensity, Cartesian reordering, cuboid reshaping).

``medium``, ``source`` and ``sensor`` are dicts with the reference's field
names (``sound_speed``, ``density``, ``alpha_coeff``, ``alpha_power``,
``BonA``; ``p0``, ``p``, ``p_mask``, ``p_mode``, ``ux``/``uy``/``uz``,
``u_mask``, ``u_mode``; ``mask``, ``record``, ``record_start_index``,
``time_reversal_boundary_data``).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from .transducer import KWaveTransducer, transducer_source_datasets
from .utils import KWaveGrid, cart2grid, cart_linear_weights, reorder_binary_sensor_data, smooth

MODE = {"dirichlet": 0, "additive-no-correction": 1, "additive": 2}
PML_DEFAULT = {2: (20, 2.0), 3: (10, 2.0)}  # kspaceFirstOrder_setDefaults.m:150-167


def _as_grid(v, shape):
    v = np.asarray(v, dtype=np.float64)
    if v.size == 1:
        return v.reshape(())
    if v.shape != tuple(shape):
        raise ValueError(f"medium / source arrays must be scalars or of shape {tuple(shape)}")
    return v


def staggered_density(rho0, kgrid: KWaveGrid):
    """rho0 at x + dx/2 (etc.) by linear interpolation, original values where
    the shifted point leaves the grid (kspaceFirstOrder3D.m:583-600)."""
    rho0 = np.asarray(rho0, dtype=np.float64)
    if rho0.ndim != kgrid.dim:
        return [rho0] * kgrid.dim
    out = []
    for a in range(kgrid.dim):
        r = rho0.copy()
        lo = [slice(None)] * kgrid.dim
        hi = [slice(None)] * kgrid.dim
        lo[a] = slice(0, -1)
        hi[a] = slice(1, None)
        r[tuple(lo)] = rho0[tuple(lo)] + 0.5 * (rho0[tuple(hi)] - rho0[tuple(lo)])
        out.append(r)
    return out


def _find(mask):
    """1-based column-major indices of the non-zero entries (MATLAB find)."""
    return np.flatnonzero(np.asarray(mask).reshape(-1, order="F")) + 1


def _expand_grid(kgrid, medium, source, sensor, ps, smooth_p0, axisymmetric=False):
    """PMLInside = false: the grid grows by the PML on every side
    (kspaceFirstOrder_expandGridMatrices.m).  Medium maps extend their edge
    values, masks and p0 grow with zeros (p0 smoothed first, as
    kspaceFirstOrder_inputChecking.m:1499-1557 orders it), cuboid corners
    shift; Cartesian points keep their coordinates, which the centred grid
    preserves.  Returns the new grid, inputs and the slices that cut the
    full-grid outputs back to the user's grid (kspaceFirstOrder3DC.m:586-614).
    An axisymmetric grid grows radially at the outer radius only
    (kspaceFirstOrder_expandGridMatrices.m:40-43, 65-66)."""
    import copy

    dim = kgrid.dim
    lo = [int(p) for p in ps]
    hi = [int(p) for p in ps]
    if axisymmetric:
        lo[1] = 0
    pad = list(zip(lo, hi))
    big = KWaveGrid(tuple(n + a + b for n, a, b in zip(kgrid.N, lo, hi)), kgrid.d)
    big.set_time(kgrid.Nt, kgrid.dt)
    trim = tuple(slice(a, a + n) for a, n in zip(lo, kgrid.N))

    def grid_shaped(a):
        return np.ndim(a) == dim and tuple(np.shape(a)) == tuple(kgrid.N)

    medium = dict(medium)
    for k in ("sound_speed", "density", "alpha_coeff", "BonA"):
        if k in medium and np.size(medium[k]) > 1:
            medium[k] = np.pad(np.asarray(medium[k], dtype=np.float64), pad, mode="edge")
    expanded = {}

    def expand_transducer(tr):
        if id(tr) not in expanded:
            t = copy.deepcopy(tr)
            t.expand_grid(ps)
            expanded[id(tr)] = t
        return expanded[id(tr)]

    if isinstance(source, KWaveTransducer):
        source = expand_transducer(source)
    else:
        source = dict(source)
        if "p0" in source and np.any(np.asarray(source["p0"]) != 0):
            p0 = np.asarray(source["p0"], dtype=np.float64)
            if p0.shape != tuple(kgrid.N):
                raise ValueError("source.p0 must be the same size as the computational grid.")
            if smooth_p0:
                p0 = smooth(_mirror_wswa(p0), True)[:, :p0.shape[1]] if axisymmetric else smooth(p0, True)
            source["p0"] = np.pad(p0, pad)
        for k in ("p_mask", "u_mask"):
            if k in source:
                source[k] = np.pad(np.asarray(source[k]), pad)
    if isinstance(sensor, KWaveTransducer):
        sensor = expand_transducer(sensor)
    else:
        sensor = dict(sensor)
        mask = np.asarray(sensor["mask"])
        if grid_shaped(mask) and not (mask.ndim == 2 and mask.shape[0] == 2 * dim and dim == 3):
            sensor["mask"] = np.pad(mask, pad)
        elif mask.ndim == 2 and mask.shape[0] == 2 * dim:
            sh = np.asarray(lo * 2)[:, None]
            sensor["mask"] = np.asarray(mask, dtype=np.int64) + sh
    return big, medium, source, sensor, trim


def prepare(kgrid: KWaveGrid, medium: dict, source: dict, sensor: dict, *, pml_size=None,
            pml_alpha=None, pml_inside=True, smooth_p0=True, data_cast="single", cart_interp="nearest",
            axisymmetric=False):
    """Build the datasets of the HDF5 input file (saveToDisk.m:44-378)
    plus the record list / start index the wrapper turns into flags.

    ``cart_interp`` is the reference's 'CartInterp' for Cartesian sensor
    points: "nearest" maps them to grid points, the only form an input file
    can hold (kspaceFirstOrder_saveToDisk.m:35-37); "linear" passes each
    point's simplex vertices and barycentric weights
    (``sensor_interp_index`` / ``sensor_interp_weight``) and the solver
    interpolates every step (the in-memory solvers' default,
    kspaceFirstOrder_extractSensorData.m:296-420).

    ``axisymmetric`` is kspaceFirstOrderAS: a 2D grid with x axial and y
    radial (the axis on the first row of y); absorption is Stokes
    (kspaceFirstOrder_inputChecking.m:172-199).

    Returns (inp, record, start_index, meta)."""
    if cart_interp not in ("nearest", "linear"):
        raise ValueError("cart_interp must be 'nearest' or 'linear'")
    if axisymmetric:
        if kgrid.dim != 2:
            raise ValueError("axisymmetric simulations need a 2D grid")
        if isinstance(source, KWaveTransducer) or isinstance(sensor, KWaveTransducer):
            raise ValueError("Transducer inputs are only compatible with 3D simulations.")
        if "uy" in source:
            raise NotImplementedError("radial velocity sources are not supported for axisymmetric simulations")
    dim = kgrid.dim
    if kgrid.dt is None or kgrid.Nt is None:
        kgrid.make_time(medium["sound_speed"])
    size_def, alpha_def = PML_DEFAULT[dim]
    ps = np.broadcast_to(np.asarray(size_def if pml_size is None else pml_size, dtype=int), (dim,))
    pa = np.broadcast_to(np.asarray(alpha_def if pml_alpha is None else pml_alpha, dtype=float), (dim,))
    trim = None
    if not pml_inside:
        kgrid, medium, source, sensor, trim = _expand_grid(kgrid, medium, source, sensor, ps, smooth_p0,
                                                           axisymmetric)
        smooth_p0 = False  # smoothed on the user's grid, before the expansion
    shape = kgrid.N
    # a transducer replaces the source struct, or serves as the sensor:
    # pressure at its active grid points, averaged per element afterwards
    # (kspaceFirstOrder3DC.m:780-783)
    tr_source = source if isinstance(source, KWaveTransducer) else None
    tr_sensor = sensor if isinstance(sensor, KWaveTransducer) else None
    source = {} if tr_source is not None else dict(source)
    if tr_sensor is not None:
        sensor = {"mask": tr_sensor.active_elements_mask, "record_start_index": tr_sensor.record_start_index}
    sensor = dict(sensor)
    meta = {"dim": dim, "time_rev": False, "cuboid": False, "reorder_index": None, "transducer": tr_sensor,
            "trim": trim}

    # time reversal -> dirichlet pressure source (kspaceFirstOrder3DC.m:437-459)
    if "time_reversal_boundary_data" in sensor:
        source = {"p_mask": sensor["mask"], "p": np.fliplr(np.asarray(sensor["time_reversal_boundary_data"])),
                  "p_mode": "dirichlet"}
        sensor = {"mask": np.ones(shape), "record": ["p_final"]}
        meta["time_rev"] = True

    c0 = _as_grid(medium["sound_speed"], shape)
    rho0 = _as_grid(medium.get("density", 1.0), shape)
    c_ref = medium.get("sound_speed_ref", None)
    if c_ref is None or c_ref == "max":
        c_ref = float(np.max(c0))  # kspaceFirstOrder_setSoundSpeedRef.m:28-47
    elif c_ref == "min":
        c_ref = float(np.min(c0))
    elif c_ref == "mean":
        c_ref = float(np.mean(c0))
    inp = {
        "Nx": kgrid.Nx, "Ny": kgrid.Ny, "Nz": kgrid.Nz, "Nt": kgrid.Nt,
        "dx": kgrid.dx, "dy": kgrid.dy, "dz": kgrid.dz, "dt": kgrid.dt, "c_ref": c_ref,
        "pml_x_size": int(ps[0]), "pml_y_size": int(ps[1]), "pml_z_size": int(ps[2]) if dim == 3 else 0,
        "pml_x_alpha": float(pa[0]), "pml_y_alpha": float(pa[1]),
        "pml_z_alpha": float(pa[2]) if dim == 3 else 0.0,
        "c0": c0, "rho0": rho0,
    }
    for name, r in zip(("rho0_sgx", "rho0_sgy", "rho0_sgz"), staggered_density(rho0, kgrid)):
        inp[name] = r
    if "BonA" in medium:
        inp["nonlinear_flag"] = 1
        inp["BonA"] = _as_grid(medium["BonA"], shape)
    if "alpha_coeff" in medium:
        stokes = medium.get("alpha_mode") == "stokes" or axisymmetric
        y = 2.0 if stokes else float(medium["alpha_power"])
        if not stokes and y == 1.0:
            raise ValueError("medium.alpha_power = 1 is not supported (the dispersion term is singular)")
        inp["absorbing_flag"] = 2 if stokes else 1
        inp["alpha_coeff"] = _as_grid(medium["alpha_coeff"], shape)
        inp["alpha_power"] = y

    # initial pressure (kspaceFirstOrder_inputChecking.m:746-783, 1499-1553)
    if "p0" in source and np.any(np.asarray(source["p0"]) != 0):
        p0 = np.asarray(source["p0"], dtype=np.float64)
        if p0.shape != tuple(shape):
            raise ValueError("source.p0 must be the same size as the computational grid.")
        if smooth_p0 and axisymmetric:
            # smoothed on the mirrored grid (kspaceFirstOrder_inputChecking.m:1504-1533)
            p0 = smooth(_mirror_wswa(p0), True)[:, :shape[1]]
        elif smooth_p0:
            p0 = smooth(p0, True)
        inp["p0_source_flag"] = 1
        inp["p0_source_input"] = p0
    # pressure source (inputChecking.m:786-893, scaleSourceTerms.m:50-128)
    if "p" in source:
        mask = np.asarray(source["p_mask"])
        pos = _find(mask)
        sig = np.atleast_2d(np.asarray(source["p"], dtype=np.float64)).copy()
        labels = np.unique(mask)
        labelled = not (labels.size <= 2 and labels.sum() == 1)
        mode = source.get("p_mode", "additive")
        if "p_frequency_ref" in source:
            sig = sig * np.cos(2 * np.pi * source["p_frequency_ref"] * kgrid.dt / 2)
            mode = "additive-no-correction"
        # row r of the signal matrix is scaled with c0 at the r-th source
        # position, as the reference's loop over rows does
        c_at = (lambda i: float(c0)) if c0.size == 1 else (lambda i: float(c0.reshape(-1, order="F")[i - 1]))
        for r in range(sig.shape[0]):
            c = c_at(pos[r])
            if mode == "dirichlet":
                sig[r] = sig[r] / (dim * c ** 2)
            else:
                sig[r] = sig[r] * (2 * kgrid.dt / (dim * c * kgrid.dx))
        if labelled:
            # one signal per label -> one signal per source point
            lab = np.asarray(mask).reshape(-1, order="F")[pos - 1].astype(int)
            sig = sig[lab - 1]
        inp.update(p_source_flag=sig.shape[1], p_source_mode=MODE[mode],
                   p_source_many=int(sig.shape[0] > 1), p_source_index=pos, p_source_input=sig)
    # velocity sources (inputChecking.m:896-1011, scaleSourceTerms.m:285-369)
    comps = [c for c in "xyz"[:dim] if "u" + c in source]
    if comps:
        mask = np.asarray(source["u_mask"])
        pos = _find(mask)
        mode = source.get("u_mode", "additive")
        many = 0
        for i, c in enumerate("xyz"[:dim]):
            if "u" + c not in source:
                continue
            sig = np.atleast_2d(np.asarray(source["u" + c], dtype=np.float64)).copy()
            many = int(sig.shape[0] > 1)
            if "u_frequency_ref" in source:
                sig = sig * np.cos(2 * np.pi * source["u_frequency_ref"] * kgrid.dt / 2)
            if mode != "dirichlet":
                for r in range(sig.shape[0]):
                    cc = float(c0) if c0.size == 1 else float(c0.reshape(-1, order="F")[pos[r] - 1])
                    sig[r] = sig[r] * (2 * cc * kgrid.dt / kgrid.d[i])
            inp[f"u{c}_source_flag"] = sig.shape[1]
            inp[f"u{c}_source_input"] = sig
        if "u_frequency_ref" in source:
            mode = "additive-no-correction"
        inp.update(u_source_mode=MODE[mode], u_source_many=many, u_source_index=pos)
    if tr_source is not None:
        if dim != 3:
            raise ValueError("Transducer inputs are only compatible with 3D simulations.")
        inp.update(transducer_source_datasets(tr_source, c0, kgrid))

    # sensor (inputChecking.m:502-634, 1606-1659; 3DC.m:425-431)
    mask = np.asarray(sensor["mask"])
    record = list(sensor.get("record", ["p"]))
    if mask.shape == tuple(shape) and not (mask.ndim == 2 and mask.shape[0] == 2 * dim and dim == 3):
        inp["sensor_mask_type"] = 0
        inp["sensor_mask_index"] = _find(mask)
    elif mask.ndim == 2 and mask.shape[0] == 2 * dim:
        corners = np.asarray(mask, dtype=np.int64)
        if dim == 2:
            c6 = np.ones((6, corners.shape[1]), dtype=np.int64)
            c6[0], c6[1], c6[3], c6[4] = corners[0], corners[1], corners[2], corners[3]
            corners = c6
        inp["sensor_mask_type"] = 1
        inp["sensor_mask_corners"] = corners
        meta["cuboid"] = True
        meta["corners"] = corners
    elif mask.ndim == 2 and mask.shape[0] == dim and cart_interp == "linear":
        # Cartesian points, linear interpolation: the solver records the
        # vertices of the simplex around each point and forms the point
        # every step (kspaceFirstOrder_extractSensorData.m:296-420)
        verts, w = cart_linear_weights(kgrid, mask)
        inp["sensor_mask_type"] = 0
        inp["sensor_interp_index"] = verts
        inp["sensor_interp_weight"] = w
        meta["interp"] = True
    elif mask.ndim == 2 and mask.shape[0] == dim:
        # Cartesian points: nearest-neighbour mapping, as the file path requires
        # (kspaceFirstOrder_saveToDisk.m:35-37; createStorageVariables.m:33-51)
        bmask, _, reorder_index = cart2grid(kgrid, mask)
        inp["sensor_mask_type"] = 0
        inp["sensor_mask_index"] = _find(bmask)
        meta["reorder_index"] = reorder_index
    else:
        raise ValueError("sensor.mask must be a binary grid, cuboid corners or Cartesian points")
    if any(r in record for r in ("I", "I_avg")):
        record = [r for r in record if r not in ("I", "I_avg")] + [r for r in ("u_non_staggered", "p")
                                                                   if r not in record]
        meta["intensity"] = [r for r in sensor["record"] if r in ("I", "I_avg")]
    if axisymmetric:
        if meta.get("reorder_index") is not None or meta.get("interp"):
            raise NotImplementedError("Cartesian sensor masks are not supported for axisymmetric simulations")
        if any(r in record for r in ("u_non_staggered", "I", "I_avg")):
            raise NotImplementedError("u_non_staggered and intensity are not supported for axisymmetric simulations")
        inp["axisymmetric_flag"] = 1
    start = int(sensor.get("record_start_index", 1))
    meta["user_record"] = list(sensor.get("record", ["p"]))
    meta["has_record"] = "record" in sensor
    return inp, record, start, meta


def _mirror_wswa(a):
    """The 'WSWA-FFT' radial mirror of a field on the pressure points:
    columns [a, 0, -flip(a[:, 1:]), -a, 0, flip(a[:, 1:])]
    (kspaceFirstOrderAS.m:711-714)."""
    a = np.asarray(a, dtype=np.float64)
    ny = a.shape[1]
    out = np.zeros((a.shape[0], 4 * ny))
    out[:, :ny] = a
    out[:, ny + 1:2 * ny] = -a[:, 1:][:, ::-1]
    out[:, 2 * ny:3 * ny] = -a
    out[:, 3 * ny + 1:] = a[:, 1:][:, ::-1]
    return out


def fourier_shift(data, shift, axis=-1):
    """fourierShift.m along `axis`."""
    data = np.asarray(data, dtype=np.float64)
    N = data.shape[axis]
    if N % 2 == 0:
        k = 2 * np.pi * np.arange(-N // 2, N // 2) / N
    else:
        k = 2 * np.pi * np.arange(-(N - 1) // 2, (N - 1) // 2 + 1) / N
    k[N // 2] = 0
    sh = [1] * data.ndim
    sh[axis] = -1
    op = np.fft.ifftshift(np.exp(1j * k * shift)).reshape(sh)
    return np.real(sfft.ifft(op * sfft.fft(data, axis=axis), axis=axis))


def postprocess(out: dict, inp: dict, meta: dict):
    """Intensity, Cartesian reorder and cuboid reshape
    (kspaceFirstOrder_saveIntensity.m:42-75, _reorderCartData.m,
    _reorderCuboidCorners.m:33-272)."""
    dim = meta["dim"]
    if meta.get("trim") is not None:
        for k in list(out):
            if k.endswith("_all") or k.endswith("_final"):
                out[k] = out[k][meta["trim"]]
    if meta.get("intensity"):
        for c in "xyz"[:dim]:
            u_sgt = fourier_shift(out[f"u{c}_non_staggered"], 0.5, axis=-1)
            out["I" + c] = out["p"] * u_sgt
            if "I_avg" in meta["intensity"]:
                out[f"I{c}_avg"] = np.mean(out["I" + c], axis=-1)
        if "I" not in meta["intensity"]:
            for c in "xyz"[:dim]:
                out.pop("I" + c, None)
        if "u_non_staggered" not in meta["user_record"]:
            for c in "xyz"[:dim]:
                out.pop(f"u{c}_non_staggered", None)
        if "p" not in meta["user_record"]:
            out.pop("p", None)
    if meta.get("reorder_index") is not None:
        for k in list(out):
            if not (k.endswith("_all") or k.endswith("_final")):
                out[k] = reorder_binary_sensor_data(out[k], meta["reorder_index"])
    if meta.get("cuboid"):
        corners = meta["corners"]
        res = []
        start = 0
        for k in range(corners.shape[1]):
            sz = tuple(int(corners[3 + a, k] - corners[a, k] + 1) for a in range(dim))
            n = int(np.prod(sz))
            item = {}
            for key, v in out.items():
                if key.endswith("_all") or key.endswith("_final"):
                    item[key] = v
                    continue
                seg = v[start:start + n]
                item[key] = seg.reshape(sz + ((seg.shape[1],) if seg.ndim == 2 else ()), order="F")
            res.append(item)
            start += n
        return res
    if meta.get("transducer") is not None:
        out["p"] = meta["transducer"].combine_sensor_data(out["p"])
    if meta["time_rev"]:
        return out["p_final"]
    if not meta["has_record"]:
        return out["p"]
    return out


def kspace_first_order(kgrid: KWaveGrid, medium: dict, source: dict, sensor: dict, *, device=-1, **options):
    """Run a simulation (the G-suffixed drop-in path) and return sensor_data
    as the reference does."""
    from . import _lib  # the CUDA library is mapped here, on the first solve

    inp, record, start, meta = prepare(kgrid, medium, source, sensor, **options)
    out = _lib.solve(inp, record=record, start_index=start, device=device)
    return postprocess(out, inp, meta)


kspaceFirstOrder2D = kspace_first_order
kspaceFirstOrder3D = kspace_first_order


def kspaceFirstOrderAS(kgrid: KWaveGrid, medium: dict, source: dict, sensor: dict, *, device=-1, **options):
    """The axisymmetric solver (kspaceFirstOrderAS.m): x axial, y radial."""
    return kspace_first_order(kgrid, medium, source, sensor, device=device, axisymmetric=True, **options)
