"""ORACLE -- test infrastructure only, never the product path.

A NumPy restatement of ac-fdtd's reference solver ``AcousticFDTD`` (``src/ac_fdtd/scheme.py``)
and of the host setup it calls (``grid.py``, ``boundaries.py``, ``air.py``), written as plain
array passes in the reference's operation order so that it reproduces the reference's float64
and float32 arithmetic. It is the checker for the CUDA backend: only ``tests/``, the smoke test
and ``bench.py``'s CPU baseline may import it.

Parity of this restatement with the reference itself is pinned by ``tests/golden/`` fixtures
that ``tests/golden/make_golden.py`` generated by running the reference.

Inputs are read by attribute (``grid.dx/nx/ny/nz``, ``walls.values``, the layer's
``thickness/target_reflection/order/faces``, the air's ``temperature/relative_humidity/
static_pressure/classical/relaxation``), so this module depends on neither the product package
nor the reference.
"""

from __future__ import annotations

import math

import numpy as np

__all__ = [
    "OracleFDTD",
    "oracle_processes",
    "oracle_wall_list",
    "oracle_layer_factors",
    "oracle_cell_index",
    "FACES",
]

FACES = ((0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1))  # boundaries.py:73


def oracle_cell_index(dx, shape, point):
    """grid.py:131-147 -- floor(x/dx + 1e-6) clipped to the grid."""
    return tuple(
        int(min(max(math.floor(x / dx + 1e-6), 0), n - 1)) for x, n in zip(point, shape, strict=True)
    )


def oracle_processes(air, sound_speed, dt):
    """air.py:137-218 -- (strength, relaxation_time) of O2, N2 and the Nyquist classical term."""
    kelvin = air.temperature + 273.15
    pa = air.static_pressure / 101325.0
    tr = kelvin / 293.15
    exponent = -6.8346 * (273.16 / kelvin) ** 1.261 + 4.6151
    h = air.relative_humidity * 10.0**exponent / pa
    f_o = pa * (24.0 + 4.04e4 * h * (0.02 + h) / (0.391 + h))
    f_n = pa * tr**-0.5 * (9.0 + 280.0 * h * math.exp(-4.170 * (tr ** (-1 / 3) - 1.0)))
    classical = 1.84e-11 / pa * tr**0.5
    oxygen = tr**-2.5 * 0.01275 * math.exp(-2239.1 / kelvin)
    nitrogen = tr**-2.5 * 0.1068 * math.exp(-3352.0 / kelvin)
    out = []
    if air.relaxation:
        for coefficient, fr in ((oxygen, f_o), (nitrogen, f_n)):
            out.append((coefficient * sound_speed / math.pi, 1.0 / (2.0 * math.pi * fr)))
    if air.classical:
        nyquist = 0.5 / dt
        out.append((classical * nyquist * sound_speed / math.pi, 1.0 / (2.0 * math.pi * nyquist)))
    return out


def oracle_wall_list(shape, sound_speed, dt, dx, xi):
    """boundaries.py:167-207 -- sorted flat indices of wall cells and their summed ``a``."""
    strides = (shape[1] * shape[2], shape[2], 1)
    scale = sound_speed * dt / (2.0 * dx)
    flats, values = [], []
    for (axis, side), value in zip(FACES, xi, strict=True):
        if value == 0.0:
            continue
        ranges = [np.arange(n) for n in shape]
        ranges[axis] = np.array([0 if side == 0 else shape[axis] - 1])
        grids = np.meshgrid(*ranges, indexing="ij")
        flat = sum(g * s for g, s in zip(grids, strides, strict=True)).ravel().astype(np.int64)
        flats.append(flat)
        values.append(np.full(flat.size, scale * value))
    if not flats:
        return np.empty(0, dtype=np.int64), np.empty(0)
    flat = np.concatenate(flats)
    coefficient = np.concatenate(values)
    unique, inverse = np.unique(flat, return_inverse=True)
    summed = np.zeros(unique.size)
    np.add.at(summed, inverse, coefficient)
    return unique, summed


def oracle_layer_factors(shape, dx, sound_speed, dt, layer):
    """boundaries.py:238-283 -- per-axis exp(-sigma dt) at cell centres and at faces."""
    depth = layer.thickness * dx
    sigma_max = -(layer.order + 1.0) * sound_speed * math.log(layer.target_reflection) / (2.0 * depth)
    faces = tuple(tuple(f) for f in layer.faces)

    def factors(x, extent, axis):
        distance = np.full(x.shape, np.inf)
        if (axis, 0) in faces:
            distance = np.minimum(distance, x)
        if (axis, 1) in faces:
            distance = np.minimum(distance, extent - x)
        inside = np.clip(1.0 - distance / depth, 0.0, 1.0)
        return np.exp(-sigma_max * inside**layer.order * dt)

    cells = [factors((np.arange(n) + 0.5) * dx, n * dx, a) for a, n in enumerate(shape)]
    faces_ = [factors(np.arange(n + 1) * dx, n * dx, a) for a, n in enumerate(shape)]
    return cells, faces_


def _slabs(factor, axis):
    """boundaries.py:286-318 -- the leading and trailing runs where the factor is below one."""
    damping = factor < 1.0
    if not damping.any():
        return []

    def at(span):
        return tuple(span if a == axis else slice(None) for a in range(3))

    def shaped(v):
        s = [1, 1, 1]
        s[axis] = -1
        return v.reshape(s)

    if damping.all():
        return [(at(slice(None)), shaped(factor))]
    lead = int(np.argmin(damping)) if damping[0] else 0
    trail = int(np.argmin(damping[::-1])) if damping[-1] else 0
    out = []
    if lead:
        out.append((at(slice(0, lead)), shaped(factor[:lead])))
    if trail:
        out.append((at(slice(factor.size - trail, None)), shaped(factor[factor.size - trail:])))
    return out


def _hi(axis):
    return tuple(slice(1, None) if a == axis else slice(None) for a in range(3))


def _lo(axis):
    return tuple(slice(None, -1) if a == axis else slice(None) for a in range(3))


def _inner(axis):
    return tuple(slice(1, -1) if a == axis else slice(None) for a in range(3))


class OracleFDTD:
    """scheme.py:82-389 restated: same constructor arguments, same state, same step order."""

    def __init__(self, grid, medium, courant=1.0, dtype=np.float64, walls=None,
                 absorbing_layer=None, air_absorption=None):
        if not 0.0 < courant <= 1.0:
            raise ValueError(f"courant must be in (0, 1], got {courant}")
        self.grid = grid
        self.medium = medium
        self.dtype = dt_ = np.dtype(dtype)
        self.shape = shape = (int(grid.nx), int(grid.ny), int(grid.nz))
        dx = self.dx = float(grid.dx)
        c = float(medium.sound_speed)
        rho = float(medium.density)
        self.dt = dt = courant * (dx / (c * math.sqrt(3)))          # grid.py:37-45, scheme.py:127
        self.step_index = 0
        self.p = np.zeros(shape, dtype=dt_)
        self.velocity = []
        for axis in range(3):
            s = list(shape)
            s[axis] += 1
            self.velocity.append(np.zeros(s, dtype=dt_))
        self.cv = dt_.type(dt / (rho * dx))                        # scheme.py:135
        self.cp = dt_.type(rho * c**2 * dt / dx)                   # scheme.py:136-138
        self.cs = dt_.type(rho * c**2 * dt)                        # scheme.py:141
        xi = tuple(walls.values) if walls is not None else (0.0,) * 6
        index, a = oracle_wall_list(shape, c, dt, dx, xi)          # scheme.py:154-157
        self.wall_index = index
        self.wall_fu = (1.0 / (1.0 + a)).astype(dt_)
        self.wall_fp = (a / (1.0 + a)).astype(dt_)
        self.relax = []                                            # scheme.py:164-191
        if air_absorption is not None:
            processes = oracle_processes(air_absorption, c, dt)
            relaxed = c**2 / (1.0 + sum(strength for strength, _ in processes))
            for strength, tau in processes:
                decay = math.exp(-dt / tau)
                mean_weight = (tau / dt) * (1.0 - decay)
                gain = rho * relaxed * strength / dx
                self.relax.append([np.zeros(shape, dtype=dt_), dt_.type(decay),
                                   dt_.type(dt * mean_weight), dt_.type(gain)])
        self.relax_scale = dt_.type(dt * sum(r[3] for r in self.relax))
        self.p_slabs = []
        self.v_slabs = [[], [], []]
        if absorbing_layer is not None:                            # scheme.py:194-212
            cells, faces = oracle_layer_factors(shape, dx, c, dt, absorbing_layer)
            self.p_slabs = [s for a in range(3) for s in _slabs(cells[a].astype(dt_), a)]
            for comp in range(3):
                self.v_slabs[comp] = [
                    s for a in range(3)
                    for s in _slabs((faces[a] if a == comp else cells[a]).astype(dt_), a)
                ]
        self.sources = []
        self.receivers = []

    @property
    def time(self):
        return self.step_index * self.dt

    def add_volume_source(self, point, signal):                   # scheme.py:231-244
        self.sources.append((oracle_cell_index(self.dx, self.shape, point),
                             np.asarray(signal, dtype=self.dtype)))

    def add_pressure_receiver(self, point):                       # scheme.py:246-255
        self.receivers.append((oracle_cell_index(self.dx, self.shape, point), []))
        return len(self.receivers) - 1

    @property
    def recorded_pressure(self):                                  # scheme.py:257-262
        if not self.receivers:
            return np.zeros((0, 0))
        return np.array([samples for _, samples in self.receivers])

    def step(self):                                               # scheme.py:285-296
        p, v = self.p, self.velocity
        for axis in range(3):                                     # scheme.py:307-311
            v[axis][_inner(axis)] -= self.cv * (p[_hi(axis)] - p[_lo(axis)])
        for comp in range(3):
            for index, factor in self.v_slabs[comp]:
                v[comp][index] *= factor
        flat = p.reshape(-1)                                      # scheme.py:313-335
        previous = flat[self.wall_index].copy() if self.wall_index.size else None
        div = np.subtract(v[0][_hi(0)], v[0][_lo(0)])
        for axis in (1, 2):
            div += np.subtract(v[axis][_hi(axis)], v[axis][_lo(axis)])
        for state, decay, mean, gain in self.relax:               # scheme.py:337-358
            target = div * gain
            offset = state - target
            np.multiply(offset, decay, out=state)
            state += target
            p += offset * mean
        if self.relax:
            p += div * self.relax_scale
        p -= div * self.cp
        if previous is not None:
            flat[self.wall_index] = flat[self.wall_index] * self.wall_fu - previous * self.wall_fp
        for index, factor in self.p_slabs:                         # scheme.py:292
            p[index] *= factor
        for index, signal in self.sources:                        # scheme.py:360-363
            if self.step_index < len(signal):
                p[index] += self.cs * signal[self.step_index]
        self.step_index += 1
        for index, samples in self.receivers:
            samples.append(p[index])

    def run(self, n):
        for _ in range(n):
            self.step()

    def energy(self):                                             # scheme.py:365-389
        rho = float(self.medium.density)
        c = float(self.medium.sound_speed)
        p = self.p
        potential = float(np.dot(p.ravel(), p.ravel())) / (2.0 * rho * c**2)
        kinetic = coupling = 0.0
        for axis in range(3):
            comp = self.velocity[axis]
            kinetic += 0.5 * rho * float(np.dot(comp.ravel(), comp.ravel()))
            gradient = (p[_hi(axis)] - p[_lo(axis)]) / self.dx
            coupling += float(np.sum(comp[_inner(axis)] * gradient))
        return self.dx**3 * (potential + kinetic - 0.5 * self.dt * coupling)
