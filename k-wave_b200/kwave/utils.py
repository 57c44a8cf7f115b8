"""Host-side restatements of the reference's MATLAB helper functions that
build and pre-process simulation inputs (these run in MATLAB before the
drop-in binary is called, so they are host code here too, in FP64).

Each function cites the reference file it follows.  Arrays use MATLAB axis
order, shape (Nx, Ny[, Nz]).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft


def matlab_round(x):
    """MATLAB round(): halves away from zero."""
    x = np.asarray(x, dtype=np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def colon(a, step, b):
    """MATLAB a:step:b for floats (element count with the colon tolerance)."""
    n = int(np.floor((b - a) / step * (1 + 4 * np.finfo(float).eps) + 1e-10)) + 1
    return a + step * np.arange(max(n, 0))


# ---------------------------------------------------------------------------
# grid (k-Wave/kWaveGrid.m)
# ---------------------------------------------------------------------------
def make_dim(n: int, d: float) -> np.ndarray:
    """Centred wavenumber vector (kWaveGrid.m:779-797)."""
    if n % 2 == 0:
        nx = np.arange(-n // 2, n // 2) / n
    else:
        nx = np.arange(-(n - 1) // 2, (n - 1) // 2 + 1) / n
    nx[n // 2] = 0.0
    return (2.0 * np.pi / d) * nx


class KWaveGrid:
    """The parts of kWaveGrid used by the fluid solvers (kWaveGrid.m:340-433,
    493-531, 612-669)."""

    def __init__(self, N, d):
        self.N = tuple(int(n) for n in N)
        self.d = tuple(float(v) for v in d)
        self.dim = len(self.N)
        self.kvec = [make_dim(n, dd) for n, dd in zip(self.N, self.d)]
        self.Nt = None
        self.dt = None

    @property
    def Nx(self):
        return self.N[0]

    @property
    def Ny(self):
        return self.N[1]

    @property
    def Nz(self):
        return self.N[2] if self.dim == 3 else 1

    @property
    def dx(self):
        return self.d[0]

    @property
    def dy(self):
        return self.d[1]

    @property
    def dz(self):
        return self.d[2] if self.dim == 3 else 0.0

    def vec(self, axis):
        """x_vec / y_vec / z_vec (kWaveGrid.m:493-507)."""
        return self.N[axis] * self.d[axis] * self.kvec[axis] * self.d[axis] / (2 * np.pi)

    def set_time(self, Nt, dt):
        self.Nt, self.dt = int(Nt), float(dt)

    def make_time(self, c, cfl=0.3, t_end=None):
        """kWaveGrid.makeTime (kWaveGrid.m:612-669)."""
        c = np.asarray(c, dtype=np.float64)
        c_max, c_min = c.max(), c.min()
        if t_end is None:
            size = np.sqrt(sum((n * d) ** 2 for n, d in zip(self.N, self.d)))
            t_end = size / c_min
        self.dt = cfl * min(self.d) / c_max
        self.Nt = int(np.floor(t_end / self.dt)) + 1
        if np.floor(t_end / self.dt) != np.ceil(t_end / self.dt) and np.fmod(t_end, self.dt) == 0:
            self.Nt += 1
        return self.Nt, self.dt


# ---------------------------------------------------------------------------
# geometry (k-Wave/makeDisc.m, makeBall.m, makeCartCircle.m, makeCartSphere.m,
# cart2grid.m, private/makePixelMap.m)
# ---------------------------------------------------------------------------
def _pixel_dim(n):
    # makePixelMap.m createPixelDim, OriginSize 'single', Shift 0
    if n % 2 == 0:
        return np.arange(-n // 2 + 1, n // 2 + 1, dtype=np.float64)
    return np.arange(-(n - 1) // 2, (n - 1) // 2 + 1, dtype=np.float64)


def make_disc(Nx, Ny, cx, cy, radius):
    """makeDisc.m: binary disc of `radius` grid points centred at (cx, cy), 1-based."""
    cx = int(matlab_round(cx)) or Nx // 2 + 1
    cy = int(matlab_round(cy)) or Ny // 2 + 1
    if not (1 <= cx <= Nx and 1 <= cy <= Ny):
        raise ValueError("Disc center must be within grid.")
    x, y = np.meshgrid(_pixel_dim(Nx), _pixel_dim(Ny), indexing="ij")
    disc = (np.sqrt(x ** 2 + y ** 2) <= radius).astype(np.float64)
    return np.roll(disc, (cx - (Nx + 1) // 2, cy - (Ny + 1) // 2), axis=(0, 1))


def make_ball(Nx, Ny, Nz, cx, cy, cz, radius):
    """makeBall.m: binary ball."""
    cx = int(matlab_round(cx)) or Nx // 2 + 1
    cy = int(matlab_round(cy)) or Ny // 2 + 1
    cz = int(matlab_round(cz)) or Nz // 2 + 1
    x, y, z = np.meshgrid(_pixel_dim(Nx), _pixel_dim(Ny), _pixel_dim(Nz), indexing="ij")
    ball = (np.sqrt(x ** 2 + y ** 2 + z ** 2) <= radius).astype(np.float64)
    return np.roll(ball, (cx - (Nx + 1) // 2, cy - (Ny + 1) // 2, cz - (Nz + 1) // 2), axis=(0, 1, 2))


def make_cart_circle(radius, num_points, center=(0.0, 0.0)):
    """makeCartCircle.m (full circle): (2, num_points)."""
    angles = np.arange(num_points + 1) * 2 * np.pi / num_points + np.pi / 2
    angles = angles[:-1]
    c = np.vstack([radius * np.cos(angles), radius * np.sin(-angles)])
    c[0] += center[0]
    c[1] += center[1]
    return c


def make_cart_sphere(radius, num_points, center=(0.0, 0.0, 0.0)):
    """makeCartSphere.m (golden-section spiral): (3, num_points)."""
    inc = np.pi * (3 - np.sqrt(5))
    off = 2 / num_points
    k = np.arange(num_points)
    y = k * off - 1 + off / 2
    r = np.sqrt(1 - y ** 2)
    phi = k * inc
    s = radius * np.vstack([np.cos(phi) * r, y, np.sin(phi) * r])
    for a in range(3):
        s[a] += center[a]
    return s


def cart2grid(kgrid: KWaveGrid, cart):
    """cart2grid.m: nearest-neighbour binary mask, plus the order / reorder
    indices used to return data in the Cartesian point order."""
    cart = np.asarray(cart, dtype=np.float64)
    dim = kgrid.dim
    idx = []
    for a in range(dim):
        v = matlab_round(cart[a] / kgrid.d[a]).astype(np.int64) + kgrid.N[a] // 2 + 1
        if v.max() > kgrid.N[a] or v.min() < 1:
            raise ValueError("Cartesian points must lie within the grid defined by kgrid.")
        idx.append(v)
    grid = np.zeros(kgrid.N, dtype=np.int64)
    for j in range(cart.shape[1]):
        grid[tuple(idx[a][j] - 1 for a in range(dim))] = j + 1
    flat = grid.reshape(-1, order="F")
    reorder_index = flat[flat != 0]
    order_index = np.argsort(reorder_index, kind="stable")
    mask = (grid != 0).astype(np.float64)
    return mask, order_index, reorder_index


def cart_linear_weights(kgrid: KWaveGrid, cart):
    """Linear interpolation of Cartesian points on a triangulation of the grid:
    the cell around each point is split into triangles (2D: along the
    diagonal from its lowest to its highest corner) or the six Kuhn
    tetrahedra (3D), and the point gets the barycentric weights of the
    simplex that holds it -- exact for fields linear in x, y, z.  The
    reference triangulates the grid with MATLAB's Delaunay, which is
    degenerate on a regular grid (four co-circular points per cell), so its
    choice of diagonal can differ (kspaceFirstOrder_createStorageVariables.m:372-394,
    gridDataFast2D.m).  Returns (vertices, weights): 1-based column-major
    linear indices and weights, both (points, dim + 1)."""
    cart = np.asarray(cart, dtype=np.float64)
    dim = kgrid.dim
    n = cart.shape[1]
    f = np.empty((dim, n))
    for a in range(dim):
        f[a] = cart[a] / kgrid.d[a] + kgrid.N[a] // 2  # 0-based fractional index (x_vec of makeDim)
        if f[a].min() < -1e-9 or f[a].max() > kgrid.N[a] - 1 + 1e-9:
            raise ValueError("Cartesian points must lie within the grid defined by kgrid.")
    f = np.clip(f, 0, np.array(kgrid.N, dtype=np.float64)[:, None] - 1)
    # coordinates a few ulps from a grid line (points given on grid nodes,
    # whose coordinates carry the rounding of the grid vectors) are put on
    # it, so a point on a node takes that node's value exactly
    near = np.abs(f - np.round(f)) < 1e-9
    f[near] = np.round(f[near])
    i0 = np.minimum(np.floor(f).astype(np.int64), np.array(kgrid.N)[:, None] - 2)
    t = f - i0  # in [0, 1]
    order = np.argsort(-t, axis=0, kind="stable")  # axes by decreasing fraction
    verts = np.zeros((n, dim + 1), dtype=np.int64)
    w = np.zeros((n, dim + 1))
    strides = np.cumprod([1] + list(kgrid.N[:-1]))
    for j in range(n):
        cur = i0[:, j].copy()
        ts = t[order[:, j], j]
        w[j, 0] = 1.0 - ts[0]
        verts[j, 0] = int(np.dot(cur, strides)) + 1
        for m in range(dim):
            cur[order[m, j]] += 1
            w[j, m + 1] = (ts[m] - ts[m + 1]) if m + 1 < dim else ts[m]
            verts[j, m + 1] = int(np.dot(cur, strides)) + 1
    return verts, w


def reorder_binary_sensor_data(data, reorder_index):
    """reorderBinarySensorData.m: sortrows on the appended reorder index."""
    order = np.argsort(np.asarray(reorder_index), kind="stable")
    return np.asarray(data)[order]


# ---------------------------------------------------------------------------
# signals and windows (k-Wave/toneBurst.m, getWin.m, gaussian.m, smooth.m)
# ---------------------------------------------------------------------------
def _cosine_series(n, N, coeffs):
    s = coeffs[0] * np.ones_like(n, dtype=np.float64)
    for i, c in enumerate(coeffs[1:], start=1):
        s = s + (-1) ** i * c * np.cos(2 * np.pi * i * n / (N - 1))
    return s


def get_win_1d(N, kind="Blackman", param=None, symmetric=True):
    """getWin.m for 1D windows: Blackman, Tukey, Rectangular, Hanning,
    Hamming, Gaussian, Bartlett, Triangular and Cosine (getWin.m:203-247)."""
    N = int(N) + (0 if symmetric else 1)
    n = np.arange(N, dtype=np.float64)
    if kind == "Blackman":
        a = 0.16 if param is None else param
        win = _cosine_series(n, N, [(1 - a) / 2, 0.5, a / 2])
    elif kind == "Hanning":
        win = 0.5 - 0.5 * np.cos(2 * np.pi * n / (N - 1))
    elif kind == "Hamming":
        win = 0.54 - 0.46 * np.cos(2 * np.pi * n / (N - 1))
    elif kind == "Gaussian":
        g = 0.5 if param is None else param
        win = np.exp(-0.5 * ((n - (N - 1) / 2) / (g * (N - 1) / 2)) ** 2)
    elif kind == "Bartlett":
        win = 2 / (N - 1) * ((N - 1) / 2 - np.abs(n - (N - 1) / 2))
    elif kind == "Triangular":
        win = 2 / N * (N / 2 - np.abs(n - (N - 1) / 2))
    elif kind == "Cosine":
        win = np.cos(np.pi * n / (N - 1) - np.pi / 2)
    elif kind == "Tukey":
        r = 0.5 if param is None else param
        win = np.ones(N)
        index = colon(0.0, 1.0, (N - 1) * r / 2)
        rr = r * N
        m = len(index)
        win[:m] = 0.5 * (1 + np.cos(2 * np.pi / rr * (index - rr / 2)))
        win[N - m:][::-1] = win[:m]
    elif kind == "Rectangular":
        win = np.ones(N)
    else:
        raise ValueError(kind)
    if not symmetric:
        win = win[:-1]
    return win


def get_win_rotated(shape, kind="Blackman", symmetric=None):
    """getWin.m with 'Rotation' true (2D / 3D): the 1D window of the longest
    dimension evaluated at the radius, clamped at the window edge."""
    shape = tuple(int(s) for s in shape)
    if symmetric is None:
        symmetric = [True] * len(shape)
    N = np.array(shape) + np.array([0 if s else 1 for s in symmetric])
    L = int(N.max())
    win_lin = get_win_1d(L, kind)
    radius = (L - 1) / 2
    ll = np.linspace(-radius, radius, L)
    axes = [np.linspace(-radius, radius, int(n)) for n in N]
    grids = np.meshgrid(*axes, indexing="ij")
    r = np.sqrt(sum(g ** 2 for g in grids))
    r[r > radius] = radius
    win = np.interp(r, ll, win_lin)
    sl = tuple(slice(0, int(s)) for s in shape)
    return win[sl]


def smooth(mat, restore_max=False, kind="Blackman"):
    """smooth.m: multiply the spectrum by a rotated window
    (symmetric along odd dimensions), real(ifftn(fftn(mat) .* ifftshift(win)))."""
    mat = np.asarray(mat, dtype=np.float64)
    shape = mat.shape
    symmetric = [bool(s % 2) for s in shape]
    win = np.abs(get_win_rotated(shape, kind, symmetric))
    out = np.real(sfft.ifftn(sfft.fftn(mat) * np.fft.ifftshift(win)))
    if restore_max:
        out = (np.abs(mat).max() / np.abs(out).max()) * out
    return out


def gaussian(x, magnitude=None, mean=0.0, variance=1.0):
    """gaussian.m."""
    if magnitude is None:
        magnitude = (2 * np.pi * variance) ** -0.5
    return magnitude * np.exp(-((x - mean) ** 2) / (2 * variance))


def tone_burst(sample_freq, signal_freq, num_cycles, envelope="Gaussian", signal_offset=0,
               signal_length=None):
    """toneBurst.m for a single offset: returns a (1, n) signal."""
    dt = 1.0 / sample_freq
    tone_length = num_cycles / signal_freq
    tone_t = colon(0.0, dt, tone_length)
    burst = np.sin(2 * np.pi * signal_freq * tone_t)
    if envelope == "Gaussian":
        x_lim = 3
        window_x = colon(-x_lim, 2 * x_lim / (len(burst) - 1), x_lim)
        window_x = window_x[:len(burst)]
        window = gaussian(window_x, 1, 0, 1)
        burst = burst * window
        burst = burst * get_win_1d(len(burst), "Tukey", 0.05)
    elif envelope != "Rectangular":
        raise ValueError(envelope)
    n = signal_offset + len(burst) if signal_length is None else signal_length
    sig = np.zeros((1, n))
    sig[0, signal_offset:signal_offset + len(burst)] = burst
    return sig


def db2neper(alpha, y=1.0):
    """db2neper.m:50."""
    return 100 * alpha * (1e-6 / (2 * np.pi)) ** y / (20 * np.log10(np.exp(1)))
