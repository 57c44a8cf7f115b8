"""CPU oracle: a numpy/scipy restatement of k-Wave's fluid time loop.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, the
command-line binary or the ``kwave`` host package) may import or call this
module; only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline``
leg / ``--impl reference`` arm of ``bench.py`` use it, as the checker and as
the timed CPU baseline.

Parity status: UNPINNED against outputs of the reference itself.  The
reference is MATLAB (no MATLAB/Octave here) and ships no golden vectors
(regression ``.mat`` files are generated at CI time and git-ignored,
``k-Wave/testing/regression/.gitignore:2``).  The restatement is pinned
instead against the reference's own self-consistency / analytic tests
(p0 == two clicks, cuboid == binary mask, labelled == binary source,
1D/2D/3D plane-wave equivalence), restated in ``tests/test_oracle_*.py``.

The input is the set of datasets that the reference writes into the HDF5
input file of the drop-in binary (``k-Wave/private/kspaceFirstOrder_saveToDisk.m``
:44-378): pre-smoothed ``p0_source_input``, pre-scaled ``p_source_input`` /
``u*_source_input``, ``rho0_sg*`` on the staggered grids, ``c_ref``, PML
sizes/alphas, ``alpha_coeff`` in dB/(MHz^y cm).  Everything the binary must
rebuild itself (k-space operators, shift operators, PML profiles, tau/eta)
is rebuilt here in float64 and cast to the working precision, as
``kspaceFirstOrder_dataCast.m:25-110`` does for ``DataCast 'single'``.

Arrays use MATLAB axis order: shape (Nx, Ny) or (Nx, Ny, Nz); linear
indices are 1-based column-major (x fastest), i.e. ``order='F'``.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

RECORD_KEYS = (
    "p", "p_max", "p_min", "p_rms", "p_max_all", "p_min_all", "p_final",
    "u", "u_max", "u_min", "u_rms", "u_max_all", "u_min_all", "u_final",
    "u_non_staggered",
)


# ---------------------------------------------------------------------------
# grid and operators (all built in float64)
# ---------------------------------------------------------------------------

def make_dim(n: int, d: float) -> np.ndarray:
    """Wavenumber vector in centred order, ``kWaveGrid.m:779-797`` (makeDim)."""
    if n % 2 == 0:
        nx = np.arange(-n // 2, n // 2) / n
    else:
        nx = np.arange(-(n - 1) // 2, (n - 1) // 2 + 1) / n
    nx[n // 2] = 0.0
    return (2.0 * np.pi / d) * nx


def sinc(x):
    """``private/sinc.m:38-39``: sin(x)/x with the value 1 at x == 0."""
    x = np.asarray(x, dtype=np.float64)
    z = x == 0
    return np.sin(x + np.pi * z) / (x + z) + z


def get_pml(n, d, dt, c, size, alpha, staggered):
    """``private/getPML.m:49-85`` (non-axisymmetric form)."""
    pml = np.ones(n, dtype=np.float64)
    if size == 0:
        return pml
    x = np.arange(1, size + 1, dtype=np.float64)
    if staggered:
        left = alpha * (c / d) * (((x + 0.5) - size - 1) / (0 - size)) ** 4
        right = alpha * (c / d) * ((x + 0.5) / size) ** 4
    else:
        left = alpha * (c / d) * ((x - size - 1) / (0 - size)) ** 4
        right = alpha * (c / d) * (x / size) ** 4
    pml[:size] = np.exp(-left * dt / 2)
    pml[n - size:] = np.exp(-right * dt / 2)
    return pml


def db2neper(alpha, y):
    """``db2neper.m:50``."""
    return 100 * alpha * (1e-6 / (2 * np.pi)) ** y / (20 * np.log10(np.exp(1)))


def _bshape(axis, dim):
    s = [1] * dim
    s[axis] = -1
    return tuple(s)


class Operators:
    """float64 operators in FFT order (``kspaceFirstOrder3D.m:617-659``,
    ``kspaceFirstOrder_createAbsorptionVariables.m:27-99``,
    ``kspaceFirstOrder_createStorageVariables.m:85-101``)."""

    def __init__(self, inp):
        self.dim = 2 if int(inp["Nz"]) == 1 else 3
        dim = self.dim
        N = [int(inp["Nx"]), int(inp["Ny"]), int(inp["Nz"])][:dim]
        d = [float(inp["dx"]), float(inp["dy"]), float(inp.get("dz", 0.0))][:dim]
        self.N, self.d = N, d
        dt = float(inp["dt"])
        c_ref = float(inp["c_ref"])
        kvec = [np.fft.ifftshift(make_dim(N[i], d[i])) for i in range(dim)]
        self.kvec = kvec
        self.ddk_pos, self.ddk_neg, self.shift_neg = [], [], []
        for i in range(dim):
            k = kvec[i]
            self.ddk_pos.append((1j * k * np.exp(1j * k * d[i] / 2)).reshape(_bshape(i, dim)))
            self.ddk_neg.append((1j * k * np.exp(-1j * k * d[i] / 2)).reshape(_bshape(i, dim)))
            self.shift_neg.append(np.exp(-1j * k * d[i] / 2).reshape(_bshape(i, dim)))
        k2 = np.zeros(N, dtype=np.float64)
        for i in range(dim):
            k2 = k2 + (kvec[i] ** 2).reshape(_bshape(i, dim))
        self.k = np.sqrt(k2)
        self.kappa = sinc(c_ref * self.k * dt / 2)
        self.source_kappa = np.cos(c_ref * self.k * dt / 2)
        names = "xyz"
        self.pml, self.pml_sg = [], []
        for i in range(dim):
            size = int(inp[f"pml_{names[i]}_size"])
            alpha = float(inp[f"pml_{names[i]}_alpha"])
            self.pml.append(get_pml(N[i], d[i], dt, c_ref, size, alpha, False).reshape(_bshape(i, dim)))
            self.pml_sg.append(get_pml(N[i], d[i], dt, c_ref, size, alpha, True).reshape(_bshape(i, dim)))
        # absorption (kspaceFirstOrder_createAbsorptionVariables.m:27-99)
        self.absorbing = int(inp.get("absorbing_flag", 0))
        c0 = np.asarray(inp["c0"], dtype=np.float64)
        if self.absorbing == 1:
            y = float(inp["alpha_power"])
            a = db2neper(np.asarray(inp["alpha_coeff"], dtype=np.float64), y)
            with np.errstate(divide="ignore"):
                n1 = self.k ** (y - 2)
                n2 = self.k ** (y - 1)
            n1[np.isinf(n1)] = 0
            n2[np.isinf(n2)] = 0
            self.nabla1, self.nabla2 = n1, n2
            self.tau = -2 * a * c0 ** (y - 1)
            self.eta = 2 * a * c0 ** y * np.tan(np.pi * y / 2)
        elif self.absorbing == 2:
            a = db2neper(np.asarray(inp["alpha_coeff"], dtype=np.float64), 2)
            self.tau = -2 * a * c0


# ---------------------------------------------------------------------------
# sensor index helpers (bit-exact index work)
# ---------------------------------------------------------------------------

def cuboid_mask_index(corners, N):
    """Concatenated per-cuboid ``find`` (``kspaceFirstOrder_inputChecking.m:1615-1636``).

    ``corners`` is (6, K), 1-based [x1 y1 z1 x2 y2 z2] (2D files pad z with 1,
    ``kspaceFirstOrder_saveToDisk.m:365-372``).  Returns 1-based uint64 indices."""
    corners = np.asarray(corners, dtype=np.int64).reshape(6, -1)
    Nx, Ny, Nz = (list(N) + [1])[:3]
    out = []
    for k in range(corners.shape[1]):
        x1, y1, z1, x2, y2, z2 = corners[:, k]
        xs = np.arange(x1 - 1, x2)
        ys = np.arange(y1 - 1, y2)
        zs = np.arange(z1 - 1, z2)
        zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
        out.append((xx + Nx * (yy + Ny * zz)).ravel() + 1)
    return np.concatenate(out).astype(np.uint64)


def cuboid_sizes(corners):
    corners = np.asarray(corners, dtype=np.int64).reshape(6, -1)
    return [tuple(int(corners[3 + a, k] - corners[a, k] + 1) for a in range(3))
            for k in range(corners.shape[1])]


# ---------------------------------------------------------------------------
# the time loop
# ---------------------------------------------------------------------------

def simulate(inp, record=("p",), record_start_index=1, dtype=np.float32, workers=-1, on_step=None,
             max_steps=None):
    """Run the fluid time loop (``kspaceFirstOrder3D.m:767-1206``,
    ``kspaceFirstOrder2D.m:710-1042``) on HDF5-file-level inputs.

    Returns a dict of outputs in the layout of the drop-in binary's output
    file: time series as (Ns, Nt_rec), per-point reductions as (Ns,),
    ``*_all`` / ``*_final`` on the full grid (PML included).

    ``on_step(t_index)`` is called after each step and ``max_steps`` stops
    the loop early (used to time a bounded sample of a long run)."""
    record = set(record)
    for r in record:
        if r not in RECORD_KEYS:
            raise ValueError(f"unknown record option {r}")
    rdt = np.dtype(dtype)
    cdt = np.complex64 if rdt == np.float32 else np.complex128
    op = Operators(inp)
    dim, N = op.dim, op.N
    nd = tuple(N)
    Nt = int(inp["Nt"])

    def fftn(a):
        return sfft.fftn(a, workers=workers)

    def rifftn(a):
        return sfft.ifftn(a, workers=workers).real.astype(rdt, copy=False)

    def cast(a):
        a = np.asarray(a)
        if np.iscomplexobj(a):
            return a.astype(cdt)
        return a.astype(rdt)

    def field(name):
        v = np.asarray(inp[name], dtype=np.float64)
        if v.size == 1:
            return rdt.type(v.reshape(()))
        return v.reshape(nd, order="F").astype(rdt)

    dt = rdt.type(inp["dt"])
    c0 = field("c0")
    rho0 = field("rho0")
    sg_names = ["rho0_sgx", "rho0_sgy", "rho0_sgz"][:dim]
    rho0_sg_inv = [rdt.type(1) / field(n) for n in sg_names]
    kappa = cast(op.kappa)
    ddk_pos = [cast(v) for v in op.ddk_pos]
    ddk_neg = [cast(v) for v in op.ddk_neg]
    pml = [cast(v) for v in op.pml]
    pml_sg = [cast(v) for v in op.pml_sg]
    source_kappa = cast(op.source_kappa)
    nonlinear = int(inp.get("nonlinear_flag", 0)) != 0
    BonA = field("BonA") if nonlinear else None
    if op.absorbing == 1:
        nabla1, nabla2 = cast(op.nabla1), cast(op.nabla2)
        tau, eta = cast(op.tau), cast(op.eta)
    elif op.absorbing == 2:
        tau = cast(op.tau)

    def source_block(prefix):
        flag = int(inp.get(f"{prefix}_source_flag", 0))
        return flag

    # p source
    p_flag = int(inp.get("p_source_flag", 0))
    if p_flag:
        p_mode = int(inp["p_source_mode"])
        p_idx = np.asarray(inp["p_source_index"], dtype=np.int64).ravel() - 1
        p_sig = np.asarray(inp["p_source_input"], dtype=np.float64)
        p_sig = p_sig.reshape(-1, p_sig.shape[-1]).astype(rdt)
    # u sources
    u_flags = [int(inp.get(f"u{c}_source_flag", 0)) for c in "xyz"[:dim]]
    if any(u_flags):
        u_mode = int(inp["u_source_mode"])
        u_idx = np.asarray(inp["u_source_index"], dtype=np.int64).ravel() - 1
        u_sig = []
        for i, c in enumerate("xyz"[:dim]):
            if u_flags[i]:
                s = np.asarray(inp[f"u{c}_source_input"], dtype=np.float64)
                u_sig.append(s.reshape(-1, s.shape[-1]).astype(rdt))
            else:
                u_sig.append(None)
    # transducer source (kspaceFirstOrder_inputChecking.m:1155-1213): one
    # signal, a 1-based delay per point, optional apodization weights
    tr_flag = int(inp.get("transducer_source_flag", 0))
    if tr_flag:
        tr_idx = np.asarray(inp["u_source_index"], dtype=np.int64).ravel() - 1
        tr_sig = np.asarray(inp["transducer_source_input"], dtype=np.float64).ravel().astype(rdt)
        tr_delay = np.asarray(inp["delay_mask"], dtype=np.int64).ravel()
        apod = inp.get("transducer_source_apodization")
        tr_apod = rdt(1) if apod is None else np.asarray(apod, dtype=np.float64).ravel().astype(rdt)
        if tr_delay.min() < 1 or tr_delay.max() - 1 + tr_flag > tr_sig.size:
            raise ValueError("delay_mask reads past the end of transducer_source_input")
    p0_flag = int(inp.get("p0_source_flag", 0)) != 0
    if p0_flag:
        p0 = np.asarray(inp["p0_source_input"], dtype=np.float64).reshape(nd, order="F").astype(rdt)

    # sensor
    mask_type = int(inp.get("sensor_mask_type", 0))
    if mask_type == 0:
        s_idx = np.asarray(inp["sensor_mask_index"], dtype=np.int64).ravel() - 1 \
            if inp.get("sensor_interp_index") is None else None
    else:
        s_idx = cuboid_mask_index(inp["sensor_mask_corners"], N).astype(np.int64) - 1
    # Cartesian points by linear interpolation: sum(field(tri) .* bc, 2)
    # every step (kspaceFirstOrder_extractSensorData.m:296-420)
    if inp.get("sensor_interp_index") is not None:
        K = dim + 1
        tri = np.asarray(inp["sensor_interp_index"], dtype=np.int64).reshape(-1, K) - 1
        bc = np.asarray(inp["sensor_interp_weight"], dtype=np.float64).reshape(-1, K)

        def at_sensors(f):
            return np.sum(f.reshape(-1, order="F")[tri] * bc, axis=1).astype(rdt)
        Ns = tri.shape[0]
    else:
        def at_sensors(f):
            return f.reshape(-1, order="F")[s_idx]
        Ns = s_idx.size
    start = int(record_start_index)
    n_rec = max(Nt - start + 1, 0)
    out = {}
    if "p" in record:
        out["p"] = np.zeros((Ns, n_rec), rdt)
    if "u" in record:
        for c in "xyz"[:dim]:
            out["u" + c] = np.zeros((Ns, n_rec), rdt)
    if "u_non_staggered" in record:
        for c in "xyz"[:dim]:
            out["u" + c + "_non_staggered"] = np.zeros((Ns, n_rec), rdt)
    for key in ("p_max", "p_min", "p_rms"):
        if key in record:
            out[key] = np.zeros(Ns, rdt)
    for key in ("u_max", "u_min", "u_rms"):
        if key in record:
            for c in "xyz"[:dim]:
                out["u" + c + key[1:]] = np.zeros(Ns, rdt)

    p = np.zeros(nd, rdt)
    rho = [np.zeros(nd, rdt) for _ in range(dim)]
    u = [np.zeros(nd, rdt) for _ in range(dim)]
    p_k = np.zeros(nd, cdt)

    def flat(a):
        return a.reshape(-1, order="F")

    def scatter_set(a, idx, vals):
        f = a.reshape(-1, order="F").copy()
        f[idx] = vals
        return f.reshape(nd, order="F")

    def scatter_add(a, idx, vals):
        f = a.reshape(-1, order="F").copy()
        f[idx] = f[idx] + vals
        return f.reshape(nd, order="F")

    def sig_at(sig, t):
        col = sig[:, t]
        return col[0] if col.shape[0] == 1 else col

    for t_index in range(1, Nt + 1):
        if max_steps is not None and t_index > max_steps:
            break
        t = t_index - 1
        # momentum conservation (kspaceFirstOrder3D.m:790-801)
        for i in range(dim):
            grad = rifftn(ddk_pos[i] * (kappa * p_k))
            u[i] = pml_sg[i] * (pml_sg[i] * u[i] - dt * rho0_sg_inv[i] * grad)
        # velocity sources (kspaceFirstOrder3D.m:804-884)
        for i in range(dim):
            if u_flags[i] >= t_index:
                v = sig_at(u_sig[i], t)
                if u_mode == 0:
                    u[i] = scatter_set(u[i], u_idx, v)
                elif u_mode == 2:
                    sm = scatter_set(np.zeros(nd, rdt), u_idx, v)
                    sm = rifftn(source_kappa * fftn(sm))
                    u[i] = u[i] + sm
                else:
                    u[i] = scatter_add(u[i], u_idx, v)
        # transducer source (kspaceFirstOrder3D.m:886-902): delay_mask advances
        # by one each step, so step t_index reads sample delay_mask + t_index - 1
        if tr_flag >= t_index:
            u[0] = scatter_add(u[0], tr_idx, tr_apod * tr_sig[tr_delay - 1 + t])
        # velocity divergence (kspaceFirstOrder3D.m:905-907)
        du = [rifftn(ddk_neg[i] * (kappa * fftn(u[i]))) for i in range(dim)]
        # mass conservation (kspaceFirstOrder3D.m:910-925)
        if not nonlinear:
            rho = [pml[i] * (pml[i] * rho[i] - dt * rho0 * du[i]) for i in range(dim)]
        else:
            rsum = rho[0] + rho[1] + (rho[2] if dim == 3 else 0)
            rho0_plus_rho = 2 * rsum + rho0
            rho = [pml[i] * (pml[i] * rho[i] - dt * rho0_plus_rho * du[i]) for i in range(dim)]
        # pressure source (kspaceFirstOrder3D.m:928-960)
        if p_flag >= t_index:
            v = sig_at(p_sig, t)
            if p_mode == 0:
                rho = [scatter_set(r, p_idx, v) for r in rho]
            elif p_mode == 2:
                sm = scatter_set(np.zeros(nd, rdt), p_idx, v)
                sm = rifftn(source_kappa * fftn(sm))
                rho = [r + sm for r in rho]
            else:
                rho = [scatter_add(r, p_idx, v) for r in rho]
        # equation of state (kspaceFirstOrder3D.m:963-1017)
        rsum = rho[0] + rho[1] + (rho[2] if dim == 3 else 0)
        if op.absorbing == 1:
            dsum = du[0] + du[1] + (du[2] if dim == 3 else 0)
            term = (rsum
                    + tau * rifftn(nabla1 * fftn(rho0 * dsum))
                    - eta * rifftn(nabla2 * fftn(rsum)))
        elif op.absorbing == 2:
            dsum = du[0] + du[1] + (du[2] if dim == 3 else 0)
            term = rsum + tau * rho0 * dsum
        else:
            term = rsum
        if nonlinear:
            term = term + BonA * rsum ** 2 / (2 * rho0)
        p = c0 ** 2 * term
        # initial pressure (kspaceFirstOrder3D.m:1021-1035, 2D.m:913-922)
        if t_index == 1 and p0_flag:
            p = p0.copy()
            rho = [p0 / (dim * c0 ** 2) for _ in range(dim)]
            p0k = fftn(p)
            u = [dt * rho0_sg_inv[i] * rifftn(ddk_pos[i] * (kappa * p0k)) / 2 for i in range(dim)]
        p_k = fftn(p)
        # sensors (kspaceFirstOrder_extractSensorData.m:39-291,462-566)
        if t_index >= start:
            fi = t_index - start + 1
            ps = at_sensors(p)
            if "p" in record:
                out["p"][:, fi - 1] = ps
            if "p_max" in record:
                out["p_max"] = ps.copy() if fi == 1 else np.maximum(out["p_max"], ps)
            if "p_min" in record:
                out["p_min"] = ps.copy() if fi == 1 else np.minimum(out["p_min"], ps)
            if "p_rms" in record:
                out["p_rms"] = np.sqrt((out["p_rms"] ** 2 * (fi - 1) + ps ** 2) / fi).astype(rdt)
            for i, c in enumerate("xyz"[:dim]):
                us = at_sensors(u[i])
                if "u" in record:
                    out["u" + c][:, fi - 1] = us
                if "u_max" in record:
                    key = "u" + c + "_max"
                    out[key] = us.copy() if fi == 1 else np.maximum(out[key], us)
                if "u_min" in record:
                    key = "u" + c + "_min"
                    out[key] = us.copy() if fi == 1 else np.minimum(out[key], us)
                if "u_rms" in record:
                    key = "u" + c + "_rms"
                    out[key] = np.sqrt((out[key] ** 2 * (fi - 1) + us ** 2) / fi).astype(rdt)
                if "u_non_staggered" in record:
                    sh = cast(op.shift_neg[i])
                    ush = sfft.ifft(sh * sfft.fft(u[i], axis=i, workers=workers), axis=i,
                                    workers=workers).real.astype(rdt)
                    out["u" + c + "_non_staggered"][:, fi - 1] = at_sensors(ush)
                if "u_max_all" in record:
                    key = "u" + c + "_max_all"
                    out[key] = u[i].copy() if fi == 1 else np.maximum(out[key], u[i])
                if "u_min_all" in record:
                    key = "u" + c + "_min_all"
                    out[key] = u[i].copy() if fi == 1 else np.minimum(out[key], u[i])
            if "p_max_all" in record:
                out["p_max_all"] = p.copy() if fi == 1 else np.maximum(out["p_max_all"], p)
            if "p_min_all" in record:
                out["p_min_all"] = p.copy() if fi == 1 else np.minimum(out["p_min_all"], p)
        if on_step is not None:
            on_step(t_index)
    if "p_final" in record:
        out["p_final"] = p
    if "u_final" in record:
        for i, c in enumerate("xyz"[:dim]):
            out["u" + c + "_final"] = u[i]
    return out


def split_cuboids(out, corners, dim, record=None):
    """Reshape flat sensor outputs into per-cuboid arrays
    (``kspaceFirstOrder_reorderCuboidCorners.m:33-272``): [cx, cy, (cz), t]."""
    sizes = cuboid_sizes(corners)
    res = []
    start = 0
    for sz in sizes:
        sz = sz[:dim] if dim == 3 else (sz[0], sz[1])
        n = int(np.prod(sz))
        item = {}
        for k, v in out.items():
            if k.endswith("_all") or k.endswith("_final"):
                continue
            seg = v[start:start + n]
            if seg.ndim == 2:
                item[k] = seg.reshape(tuple(sz) + (seg.shape[1],), order="F")
            else:
                item[k] = seg.reshape(sz, order="F")
        res.append(item)
        start += n
    return res
