"""CPU oracle for the axisymmetric fluid loop (``kspaceFirstOrderAS.m``).

TEST INFRASTRUCTURE ONLY, like ``kspace_oracle.py``: only ``tests/`` may use
it, as the checker.  Parity status: UNPINNED against outputs of the reference
(MATLAB); pinned instead against the 3D loop run on a rotationally symmetric
field (``tests/test_oracle_as.py``): two discretisations of one problem.

The restatement follows the default radial symmetry 'WSWA-FFT': each step
the pressure and velocity fields (x axial, y radial from the axis, grid
Nx x Ny) are mirrored into an Nx x 4Ny grid, even about the axis and odd
about the outer radius (``kspaceFirstOrderAS.m:709-722, 911-931``),
differentiated there with the ordinary staggered k-space operators, and cut
back to the first Ny columns.  The radial divergence carries the extra
u_r / r term (``kspaceFirstOrderAS.m:930-934``); the radial PML sits at the
outer radius only (``private/getPML.m:74-77``).  Supported: initial
pressure, pressure and axial velocity sources (dirichlet, additive,
additive without correction), lossless and Stokes media with or without
B/A, binary sensor masks recording p and u (time series, max / min / rms,
full-grid max / min / final).  Inputs are the datasets of the input file, on the Nx x Ny grid.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from .kspace_oracle import db2neper, get_pml, make_dim, sinc


def get_pml_as(n, d, dt, c, size, alpha, staggered):
    """``private/getPML.m`` with ``axisymmetric`` true: the profile at the
    far end only."""
    pml = get_pml(n, d, dt, c, size, alpha, staggered)
    pml[:size] = 1.0
    return pml


def mirror_p(a, ny):
    """The WSWA-FFT mirror of a field on the pressure grid points along y
    (axis 1): [a, 0, -flip(a[:, 1:]), -a, 0, flip(a[:, 1:])] columns
    (``kspaceFirstOrderAS.m:711-714``)."""
    out = np.zeros((a.shape[0], 4 * ny), dtype=a.dtype)
    out[:, 0:ny] = a
    out[:, ny + 1:2 * ny] = -a[:, 1:][:, ::-1]
    out[:, 2 * ny:3 * ny] = -a
    out[:, 3 * ny + 1:4 * ny] = a[:, 1:][:, ::-1]
    return out


def mirror_sg(a, ny, odd_outer=False):
    """The mirror of a field on the radially staggered points:
    [a, flip(a), -a, -flip(a)] (``kspaceFirstOrderAS.m:916-919``), or
    [a, -flip(a), -a, flip(a)] for u_r / r (``:920-923``)."""
    s = -1 if odd_outer else 1
    out = np.empty((a.shape[0], 4 * ny), dtype=a.dtype)
    out[:, 0:ny] = a
    out[:, ny:2 * ny] = s * a[:, ::-1]
    out[:, 2 * ny:3 * ny] = -a
    out[:, 3 * ny:4 * ny] = -s * a[:, ::-1]
    return out


def simulate_as(inp, record=("p",), record_start_index=1, dtype=np.float32, workers=-1):
    """Run the axisymmetric loop on file-level inputs; outputs in the layout
    of ``kspace_oracle.simulate`` (series (Ns, Nt_rec), grids (Nx, Ny))."""
    record = set(record)
    rdt = np.dtype(dtype).type
    cdt = np.complex64 if rdt == np.float32 else np.complex128
    Nx, Ny, Nt = int(inp["Nx"]), int(inp["Ny"]), int(inp["Nt"])
    dx, dy, dt = float(inp["dx"]), float(inp["dy"]), float(inp["dt"])
    c_ref = float(inp["c_ref"])
    nd = (Nx, Ny)

    def grid(name, default=None):
        v = inp.get(name, default)
        a = np.asarray(v, dtype=np.float64)
        return a.reshape(nd, order="F") if a.size > 1 else a.reshape(())

    c0 = grid("c0")
    rho0 = grid("rho0")
    rho0_sgx = grid("rho0_sgx", inp["rho0"])
    rho0_sgy = grid("rho0_sgy", inp["rho0"])
    nonlinear = int(inp.get("nonlinear_flag", 0)) != 0
    bona = grid("BonA") if nonlinear else None
    stokes = int(inp.get("absorbing_flag", 0)) == 2
    tau = -2 * db2neper(grid("alpha_coeff"), 2) * c0 if stokes else None

    # operators on the expanded grid (kspaceFirstOrderAS.m:488-519)
    kx = np.fft.ifftshift(make_dim(Nx, dx))
    ky = np.fft.ifftshift(make_dim(4 * Ny, dy))
    ddx_pos = (1j * kx * np.exp(1j * kx * dx / 2))[:, None]
    ddx_neg = (1j * kx * np.exp(-1j * kx * dx / 2))[:, None]
    ddy = (1j * ky)[None, :]
    y_pos = np.exp(1j * ky * dy / 2)[None, :]
    y_neg = np.exp(-1j * ky * dy / 2)[None, :]
    k = np.sqrt(kx[:, None] ** 2 + ky[None, :] ** 2)
    kappa = sinc(c_ref * k * dt / 2)
    source_kappa = np.cos(c_ref * k * dt / 2)
    pml_x = get_pml(Nx, dx, dt, c_ref, int(inp["pml_x_size"]), float(inp["pml_x_alpha"]), False)[:, None]
    pml_x_sg = get_pml(Nx, dx, dt, c_ref, int(inp["pml_x_size"]), float(inp["pml_x_alpha"]), True)[:, None]
    pml_y = get_pml_as(Ny, dy, dt, c_ref, int(inp["pml_y_size"]), float(inp["pml_y_alpha"]), False)[None, :]
    pml_y_sg = get_pml_as(Ny, dy, dt, c_ref, int(inp["pml_y_size"]), float(inp["pml_y_alpha"]), True)[None, :]
    y_sg = ((np.arange(Ny) + 0.5) * dy)[None, :]  # kspaceFirstOrderAS.m:570-571

    cast = lambda a: np.asarray(a, dtype=np.float64).astype(rdt)  # noqa: E731
    ddx_pos, ddx_neg, ddy, y_pos, y_neg = (a.astype(cdt) for a in (ddx_pos, ddx_neg, ddy, y_pos, y_neg))
    kappa, source_kappa = cast(kappa), cast(source_kappa)
    pml_x, pml_x_sg, pml_y, pml_y_sg = cast(pml_x), cast(pml_x_sg), cast(pml_y), cast(pml_y_sg)
    inv_y_sg = cast(1.0 / y_sg)
    c0sq, rho0f = cast(c0 ** 2), cast(rho0)
    rinv_x, rinv_y = cast(1.0 / rho0_sgx), cast(1.0 / rho0_sgy)
    bona = cast(bona) if nonlinear else None
    tau = cast(tau) if stokes else None

    fft2 = lambda a: sfft.fft2(a, workers=workers)  # noqa: E731
    ifft2r = lambda a: np.real(sfft.ifft2(a, workers=workers)).astype(rdt)  # noqa: E731

    def grad(p):
        p_k = kappa * fft2(mirror_p(p, Ny))
        return ifft2r(ddx_pos * p_k)[:, :Ny], ifft2r(ddy * y_pos * p_k)[:, :Ny]

    # sources
    p_flag = int(inp.get("p_source_flag", 0))
    if p_flag:
        p_mode = int(inp["p_source_mode"])
        p_idx = np.asarray(inp["p_source_index"], dtype=np.int64).ravel() - 1
        p_sig = np.asarray(inp["p_source_input"], dtype=np.float64)
        p_sig = p_sig.reshape(-1, p_sig.shape[-1]).astype(rdt)
    for c in "yz":
        if int(inp.get(f"u{c}_source_flag", 0)):
            raise NotImplementedError("radial velocity sources are not restated for the axisymmetric loop")
    ux_flag = int(inp.get("ux_source_flag", 0))
    if ux_flag:
        u_mode = int(inp["u_source_mode"])
        u_idx = np.asarray(inp["u_source_index"], dtype=np.int64).ravel() - 1
        ux_sig = np.asarray(inp["ux_source_input"], dtype=np.float64)
        ux_sig = ux_sig.reshape(-1, ux_sig.shape[-1]).astype(rdt)
    p0_flag = int(inp.get("p0_source_flag", 0)) != 0
    if p0_flag:
        p0 = np.asarray(inp["p0_source_input"], dtype=np.float64).reshape(nd, order="F").astype(rdt)

    s_idx = np.asarray(inp["sensor_mask_index"], dtype=np.int64).ravel() - 1
    Ns = s_idx.size
    n_rec = max(Nt - int(record_start_index) + 1, 0)
    out = {}
    if "p" in record:
        out["p"] = np.zeros((Ns, n_rec), rdt)
    if "u" in record:
        out["ux"] = np.zeros((Ns, n_rec), rdt)
        out["uy"] = np.zeros((Ns, n_rec), rdt)
    for key in ("p_max", "p_min", "p_rms"):
        if key in record:
            out[key] = np.zeros(Ns, rdt)
    for key in ("u_max", "u_min", "u_rms"):
        if key in record:
            out["ux" + key[1:]] = np.zeros(Ns, rdt)
            out["uy" + key[1:]] = np.zeros(Ns, rdt)

    def flat(a):
        return a.reshape(-1, order="F")

    def scatter(a, idx, vals, add):
        f = flat(a).copy()
        f[idx] = f[idx] + vals if add else vals
        return f.reshape(nd, order="F")

    def sig_at(sig, t):
        col = sig[:, t]
        return col[0] if col.shape[0] == 1 else col

    p = np.zeros(nd, rdt)
    rhox, rhoy = np.zeros(nd, rdt), np.zeros(nd, rdt)
    ux, uy = np.zeros(nd, rdt), np.zeros(nd, rdt)
    acc = {}
    for t_index in range(1, Nt + 1):
        t = t_index - 1
        # momentum (kspaceFirstOrderAS.m:709-780)
        dpdx, dpdy = grad(p)
        ux = pml_x_sg * (pml_x_sg * ux - dt * rinv_x * dpdx)
        uy = pml_y_sg * (pml_y_sg * uy - dt * rinv_y * dpdy)
        # axial velocity source (:785-830), mirrored like the pressure
        if ux_flag >= t_index:
            v = sig_at(ux_sig, t)
            if u_mode == 0:
                ux = scatter(ux, u_idx, v, False)
            elif u_mode == 2:
                sm = scatter(np.zeros(nd, rdt), u_idx, v, False)
                ux = ux + ifft2r(source_kappa * fft2(mirror_p(sm, Ny)))[:, :Ny]
            else:
                ux = scatter(ux, u_idx, v, True)
        # divergence with the u_r / r term (:905-935)
        duxdx = ifft2r(ddx_neg * (kappa * fft2(mirror_p(ux, Ny))))[:, :Ny]
        duydy = ifft2r(kappa * (y_neg * (ddy * fft2(mirror_sg(uy, Ny)) +
                                         fft2(mirror_sg(uy * inv_y_sg, Ny, odd_outer=True)))))[:, :Ny]
        # mass conservation (:1019-1031)
        if not nonlinear:
            rhox = pml_x * (pml_x * rhox - dt * rho0f * duxdx)
            rhoy = pml_y * (pml_y * rhoy - dt * rho0f * duydy)
        else:
            rpr = 2 * (rhox + rhoy) + rho0f
            rhox = pml_x * (pml_x * rhox - dt * rpr * duxdx)
            rhoy = pml_y * (pml_y * rhoy - dt * rpr * duydy)
        # pressure source (:1034-1079)
        if p_flag >= t_index:
            v = sig_at(p_sig, t)
            if p_mode == 0:
                rhox, rhoy = scatter(rhox, p_idx, v, False), scatter(rhoy, p_idx, v, False)
            elif p_mode == 2:
                sm = scatter(np.zeros(nd, rdt), p_idx, v, False)
                sm = ifft2r(source_kappa * fft2(mirror_p(sm, Ny)))[:, :Ny]
                rhox, rhoy = rhox + sm, rhoy + sm
            else:
                rhox, rhoy = scatter(rhox, p_idx, v, True), scatter(rhoy, p_idx, v, True)
        # equation of state (:1082-1108)
        rs = rhox + rhoy
        term = rs
        if stokes:
            term = term + tau * rho0f * (duxdx + duydy)
        if nonlinear:
            term = term + bona * rs ** 2 / (2 * rho0f)
        p = (c0sq * term).astype(rdt)
        # initial pressure (:1111-1170)
        if t_index == 1 and p0_flag:
            p = p0.copy()
            rhox = (p0 / (2 * c0sq)).astype(rdt)
            rhoy = rhox.copy()
            dpdx, dpdy = grad(p)
            ux = (dt * rinv_x * dpdx / 2).astype(rdt)
            uy = (dt * rinv_y * dpdy / 2).astype(rdt)
        # sensors (kspaceFirstOrder_extractSensorData.m with Nx x Ny fields)
        if t_index >= record_start_index:
            fi = t_index - record_start_index
            ps, uxs, uys = flat(p)[s_idx], flat(ux)[s_idx], flat(uy)[s_idx]
            if "p" in record:
                out["p"][:, fi] = ps
            if "u" in record:
                out["ux"][:, fi] = uxs
                out["uy"][:, fi] = uys
            for base, vals in (("p", (("p", ps),)), ("u", (("ux", uxs), ("uy", uys)))):
                for name, v in vals:
                    if f"{base}_max" in record:
                        out[f"{name}_max"] = v.copy() if fi == 0 else np.maximum(out[f"{name}_max"], v)
                    if f"{base}_min" in record:
                        out[f"{name}_min"] = v.copy() if fi == 0 else np.minimum(out[f"{name}_min"], v)
                    if f"{base}_rms" in record:
                        acc[name] = (v.astype(np.float64) ** 2) + (acc.get(name, 0.0) if fi else 0.0)
            for base, fields in (("p", (("p", p),)), ("u", (("ux", ux), ("uy", uy)))):
                for name, f in fields:
                    if f"{base}_max_all" in record:
                        key = f"{name}_max_all"
                        out[key] = f.copy() if fi == 0 else np.maximum(out[key], f)
                    if f"{base}_min_all" in record:
                        key = f"{name}_min_all"
                        out[key] = f.copy() if fi == 0 else np.minimum(out[key], f)
    for name, a in acc.items():
        out[f"{name}_rms"] = np.sqrt(a / n_rec).astype(rdt)
    if "p_final" in record:
        out["p_final"] = p
    if "u_final" in record:
        out["ux_final"], out["uy_final"] = ux, uy
    return out
