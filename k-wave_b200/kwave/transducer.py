"""Flat linear-array transducer: the geometry, beamforming delays and
apodization of kWaveTransducer.m, used as a source (a delayed x-velocity
source driven by one signal) or as a sensor (pressure at every grid point of
the active elements, averaged per element afterwards).

The reference class is a MATLAB handle object; this is a plain Python class
with the same property names.  Only flat transducers exist there too
(``radius`` must be infinite, kWaveTransducer.m:389-396).  Grid positions are
1-based (x, y, z) as in MATLAB; masks are arrays of the grid's shape.
"""
from __future__ import annotations

import numpy as np

from .utils import KWaveGrid, get_win_1d, matlab_round

_AUTO = "auto"


def _flat(a):
    return np.asarray(a).reshape(-1, order="F")


class KWaveTransducer:
    """kWaveTransducer.m:322-545 (constructor and masks)."""

    def __init__(self, kgrid: KWaveGrid, number_elements=128, element_width=1, element_length=20,
                 element_spacing=0, position=(1, 1, 1), radius=np.inf, active_elements=None,
                 elevation_focus_distance=np.inf, focus_distance=np.inf, steering_angle=None,
                 steering_angle_max=None, receive_apodization="Rectangular",
                 transmit_apodization="Rectangular", sound_speed=1540.0, input_signal=None):
        if kgrid.dim != 3:
            raise ValueError("Transducer inputs are only compatible with 3D simulations.")
        if kgrid.dt is None:
            raise ValueError("kgrid.dt or kgrid.t_array must be explicitly defined")
        self.stored_grid_size = tuple(int(n) for n in kgrid.N)
        self.grid_spacing = tuple(float(d) for d in kgrid.d)
        self.dt = float(kgrid.dt)
        self.number_elements = int(matlab_round(abs(number_elements)))
        self.element_width = int(matlab_round(abs(element_width)))
        self.element_length = int(matlab_round(abs(element_length)))
        self.element_spacing = int(matlab_round(abs(element_spacing)))
        self.position = [int(v) for v in matlab_round(np.abs(np.asarray(position, dtype=np.float64)))]
        if not np.isinf(radius):
            raise ValueError("Only a value of transducer.radius = inf is currently supported")
        self.radius = radius
        self.active_elements = (np.ones(self.number_elements) if active_elements is None
                                else np.asarray(active_elements, dtype=np.float64).ravel())
        self.elevation_focus_distance = float(elevation_focus_distance)
        na = self.number_active_elements
        for name, apod in (("receive", receive_apodization), ("transmit", transmit_apodization)):
            if not isinstance(apod, str) and np.size(apod) != na:
                raise ValueError(f"The length of the {name} apodization input must match the number of active "
                                 "elements")
        self.receive_apodization = receive_apodization
        self.transmit_apodization = transmit_apodization
        if not sound_speed > 0:
            raise ValueError("transducer.sound_speed must be greater than 0")
        self.sound_speed = float(sound_speed)
        self.focus_distance = float(focus_distance)
        self.record_start_index = 1
        self.stored_input_signal = None
        if input_signal is not None:
            sig = np.asarray(input_signal, dtype=np.float64)
            if sum(n > 1 for n in sig.shape) > 1:
                raise ValueError("transducer.input_signal must be a one-dimensional array")
            self.stored_input_signal = sig.ravel()
        self.stored_appended_zeros = _AUTO
        self.stored_beamforming_delays_offset = _AUTO
        self.stored_steering_angle_max = _AUTO
        self.stored_steering_angle = 0.0
        if steering_angle_max is not None:
            self.steering_angle_max = steering_angle_max
        if steering_angle is not None:
            self.steering_angle = steering_angle

        Nx, Ny, Nz = self.stored_grid_size
        px, py, pz = self.position
        w, L, s, n = self.element_width, self.element_length, self.element_spacing, self.number_elements
        if 0 in self.position:
            raise ValueError("The defined transducer must be positioned within the grid")
        if py + n * w + (n - 1) * s > Ny:
            raise ValueError("The defined transducer is too large or positioned outside the grid in the y-direction")
        if pz + L > Nz:
            raise ValueError("The defined transducer is too large or positioned outside the grid in the z-direction")
        if px > Nx:
            raise ValueError("The defined transducer is positioned outside the grid in the x-direction")
        # grid points of element e hold e; across an element the points are
        # numbered 1..element_length along z (for the elevation delays)
        self.indexed_mask = np.zeros(self.stored_grid_size, dtype=np.int64)
        self.indexed_element_voxel_mask = np.zeros(self.stored_grid_size, dtype=np.int64)
        for e in range(1, n + 1):
            y0 = py - 1 + (w + s) * (e - 1)
            self.indexed_mask[px - 1, y0:y0 + w, pz - 1:pz - 1 + L] = e
            self.indexed_element_voxel_mask[px - 1, y0:y0 + w, pz - 1:pz - 1 + L] = np.arange(1, L + 1)[None, :]

    # ------------------------------------------------------------------
    # dependent properties (kWaveTransducer.m:552-781)
    @property
    def transducer_width(self):
        return self.number_elements * self.element_width + (self.number_elements - 1) * self.element_spacing

    @property
    def number_active_elements(self):
        return int(np.sum(self.active_elements))

    @property
    def active_elements_mask(self):
        m = np.zeros(self.stored_grid_size)
        for e in range(1, self.number_elements + 1):
            m[self.indexed_mask == e] = self.active_elements[e - 1]
        return (m != 0).astype(np.float64)

    mask = active_elements_mask

    @property
    def all_elements_mask(self):
        return (self.indexed_mask != 0).astype(np.float64)

    @property
    def indexed_elements_mask(self):
        return self.indexed_mask.copy()

    @property
    def indexed_active_elements_mask(self):
        m = self.indexed_mask.copy()
        for e in range(1, self.number_elements + 1):
            if not self.active_elements[e - 1]:
                m[m == e] = 0
        lowest = int(np.flatnonzero(self.active_elements)[0]) + 1
        m[m != 0] = m[m != 0] - lowest + 1
        return m

    @property
    def steering_angle(self):
        return self.stored_steering_angle

    @steering_angle.setter
    def steering_angle(self, angle):
        angle = float(np.ravel(angle)[0])
        if not -90 < angle < 90:
            raise ValueError("Input for steering_angle must be between -90 and 90 degrees.")
        if self.stored_steering_angle_max != _AUTO and abs(angle) > self.stored_steering_angle_max:
            raise ValueError("Input for steering_angle cannot be greater than steering_angle_max.")
        self.stored_steering_angle = angle

    @property
    def steering_angle_max(self):
        return self.stored_steering_angle_max

    @steering_angle_max.setter
    def steering_angle_max(self, angle_max):
        """Fixes the zero padding and delay offset to those of the largest
        steering angle, so every angle up to it shares one signal length."""
        angle_max = float(np.ravel(angle_max)[0])
        if not -90 < angle_max < 90:
            raise ValueError("Input for steering_angle_max must be between -90 and 90.")
        if self.stored_steering_angle_max != _AUTO and abs(self.stored_steering_angle) > angle_max:
            raise ValueError("Input for steering_angle_max cannot be less than the current steering_angle.")
        self.stored_steering_angle_max = angle_max
        current = self.stored_steering_angle
        self.stored_steering_angle = angle_max
        self.stored_appended_zeros = 0
        self.stored_beamforming_delays_offset = 0
        delay_times = -self.beamforming_delays()
        max_delay, min_delay = delay_times.max(), delay_times.min()
        if not np.isinf(self.elevation_focus_distance):
            ed = self.elevation_beamforming_delays()
            max_delay += ed.max()
            min_delay += ed.min()
        self.stored_appended_zeros = int(max_delay - min_delay)
        self.stored_beamforming_delays_offset = int(-min_delay)
        self.stored_steering_angle = current

    @property
    def appended_zeros(self):
        return self.stored_appended_zeros

    @property
    def beamforming_delays_offset(self):
        return self.stored_beamforming_delays_offset

    @property
    def input_signal(self):
        """The user's signal padded with zeros for the largest delay
        (kWaveTransducer.m:552-612)."""
        sig = self.stored_input_signal
        if sig is None:
            raise ValueError("Transducer input signal is not defined")
        if self.stored_appended_zeros != _AUTO:
            z = np.zeros(int(self.stored_appended_zeros))
            return np.concatenate([z, sig, z])
        delay_max = int(np.max(self.delay_mask()))
        nz = np.flatnonzero(sig != 0)
        leading = int(nz[0]) if nz.size else sig.size
        trailing = int(sig.size - 1 - nz[-1]) if nz.size else sig.size
        if leading < delay_max + 1:
            sig = np.concatenate([np.zeros(delay_max - leading + 1), sig])
        if trailing < delay_max + 1:
            sig = np.concatenate([sig, np.zeros(delay_max - trailing + 1)])
        return sig

    # ------------------------------------------------------------------
    # methods (kWaveTransducer.m:786-1058)
    def beamforming_delays(self):
        """Per active element transmit delay in time steps (rounded)."""
        pitch = (self.element_spacing + self.element_width) * self.grid_spacing[1]
        na = self.number_active_elements
        idx = np.arange(na, dtype=np.float64) - (na - 1) / 2
        ang = self.stored_steering_angle * np.pi / 180
        if np.isinf(self.focus_distance):
            t = pitch * idx * np.sin(ang) / self.sound_speed
        else:
            f = self.focus_distance
            t = f / self.sound_speed * (1 - np.sqrt(1 + (idx * pitch / f) ** 2 - 2 * (idx * pitch / f) * np.sin(ang)))
        return matlab_round(t / self.dt).astype(np.int64)

    def elevation_beamforming_delays(self):
        L = self.element_length
        if np.isinf(self.elevation_focus_distance):
            return np.zeros(L, dtype=np.int64)
        idx = np.arange(L, dtype=np.float64) - (L - 1) / 2
        f = self.elevation_focus_distance
        t = (f - np.sqrt((idx * self.grid_spacing[2]) ** 2 + f ** 2)) / self.sound_speed
        return -matlab_round(t / self.dt).astype(np.int64)

    def delay_mask(self, mode=None):
        """0-based index into input_signal of each active grid point at the
        first step; mode 2: elevation delays only, 3: azimuth only."""
        ia = self.indexed_active_elements_mask
        act = np.flatnonzero(_flat(ia))
        m = np.zeros(int(np.prod(self.stored_grid_size)), dtype=np.int64)
        if (not np.isinf(self.focus_distance) or self.stored_steering_angle != 0) and mode != 2:
            dtimes = -self.beamforming_delays()
            m[act] = dtimes[_flat(ia)[act] - 1]
        if not np.isinf(self.elevation_focus_distance) and self.element_length > 1 and mode != 3:
            ed = self.elevation_beamforming_delays()
            m[act] = m[act] + ed[_flat(self.indexed_element_voxel_mask)[act] - 1]
        if self.stored_appended_zeros == _AUTO:
            m[act] = m[act] - m[act].min()
        else:
            m[act] = m[act] + self.stored_beamforming_delays_offset
        return m.reshape(self.stored_grid_size, order="F")

    def elevation_beamforming_mask(self):
        dm = _flat(self.delay_mask(2))[_flat(self.active_elements_mask) != 0]
        dm = dm - dm.min()
        mask = np.zeros((dm.size, int(dm.max()) + 1))
        mask[np.arange(dm.size), dm] = 1
        return np.fliplr(mask)

    def _apodization(self, apod):
        na = self.number_active_elements
        if not isinstance(apod, str):
            apod = np.asarray(apod, dtype=np.float64).ravel()
            if apod.size != na:
                raise ValueError("The length of the apodization input must match the number of active elements")
            return apod
        return get_win_1d(na, apod) if na > 1 else np.ones(1)

    def transmit_apodization_mask(self):
        apod = self._apodization(self.transmit_apodization)
        ia = _flat(self.indexed_active_elements_mask)
        m = np.zeros(ia.size)
        m[_flat(self.active_elements_mask) == 1] = apod[ia[ia != 0] - 1]
        return m.reshape(self.stored_grid_size, order="F")

    def expand_grid(self, expand_size):
        """Grow the grid by expand_size points on both sides of each axis
        (PMLInside = false); the elements keep their place in the medium."""
        pad = [(int(p), int(p)) for p in np.broadcast_to(np.asarray(expand_size, dtype=int), (3,))]
        self.indexed_mask = np.pad(self.indexed_mask, pad)
        self.indexed_element_voxel_mask = np.pad(self.indexed_element_voxel_mask, pad)
        self.stored_grid_size = self.indexed_mask.shape
        self.position = [p + q for p, (q, _) in zip(self.position, pad)]

    def retract_grid(self, retract_size):
        r = [int(p) for p in np.broadcast_to(np.asarray(retract_size, dtype=int), (3,))]
        sl = tuple(slice(p, n - p) for p, n in zip(r, self.stored_grid_size))
        self.indexed_mask = self.indexed_mask[sl].copy()
        self.indexed_element_voxel_mask = self.indexed_element_voxel_mask[sl].copy()
        self.stored_grid_size = self.indexed_mask.shape
        self.position = [p - q for p, q in zip(self.position, r)]

    def combine_sensor_data(self, sensor_data):
        """One series per active element from the series at each of its grid
        points (the C++ output order), shifted by the elevation delays when
        an elevation focus is set (kWaveTransducer.m:907-950)."""
        sensor_data = np.asarray(sensor_data, dtype=np.float64)
        na, w, L = self.number_active_elements, self.element_width, self.element_length
        if sensor_data.shape[0] != na * w * L:
            raise ValueError("The number of time series in the input sensor_data must match the number of grid "
                             "points in the active tranducer elements.")
        ia = _flat(self.indexed_active_elements_mask)
        ind = ia[ia > 0] - 1
        nt = sensor_data.shape[1]
        # rows follow the indexed active mask, which keeps the gaps of
        # inactive elements between active ones; MATLAB grows the output to
        # the largest index, so those gaps come back as zero rows
        out = np.zeros((max(na, int(ind.max()) + 1 if ind.size else 0), nt))
        if np.isinf(self.elevation_focus_distance):
            np.add.at(out, ind, sensor_data)
        else:
            dm = _flat(self.delay_mask(2))[_flat(self.active_elements_mask) != 0]
            for ii in range(ind.size):
                d = int(dm[ii])
                out[ind[ii], :nt - d] += sensor_data[ii, d:]
        return out * (1.0 / (w * L))

    def scan_line(self, sensor_data):
        """Delay-and-sum of per-element series into one line
        (kWaveTransducer.m:873-901); as there, elements with zero delay are
        summed without their apodization weight."""
        data = np.array(sensor_data, dtype=np.float64)
        apod = self._apodization(self.receive_apodization)
        delays = -self.beamforming_delays()
        nt = data.shape[1]
        for e in range(self.number_active_elements):
            d = int(delays[e])
            if d > 0:
                data[e] = apod[e] * np.concatenate([data[e, d:], np.zeros(d)])
            elif d < 0:
                data[e] = apod[e] * np.concatenate([np.zeros(-d), data[e, :nt + d]])
        return data.sum(axis=0)


def transducer_source_datasets(tr: KWaveTransducer, c0, kgrid: KWaveGrid):
    """The input-file datasets of a transducer source
    (kspaceFirstOrder_inputChecking.m:1155-1213, scaling
    kspaceFirstOrder_scaleSourceTerms.m:375-386, file layout
    kspaceFirstOrder_saveToDisk.m:289-293, 339-343)."""
    sig = tr.input_signal
    dmask = tr.delay_mask()
    flag = int(sig.size - np.max(dmask))
    active = _flat(tr.active_elements_mask) != 0
    if isinstance(tr.transmit_apodization, str) and tr.transmit_apodization == "Rectangular":
        apod = None
    else:
        apod = _flat(tr.transmit_apodization_mask())[active]
    pos = np.flatnonzero(active) + 1
    c0 = np.asarray(c0, dtype=np.float64)
    c = float(c0) if c0.size == 1 else float(np.mean(_flat(c0)[pos - 1]))
    sig = sig * (2 * c * kgrid.dt / kgrid.dx)
    out = {"transducer_source_flag": max(flag, 0), "u_source_index": pos,
           "delay_mask": _flat(dmask)[active].astype(np.int64) + 1, "transducer_source_input": sig}
    if apod is not None:
        out["transducer_source_apodization"] = apod
    return out
