"""Wall admittances and the graded absorbing layer, as inputs and as coefficient tables.

The value types mirror ac-fdtd ``src/ac_fdtd/boundaries.py`` (``WallAdmittances`` :120-164,
``AbsorbingLayer`` :210-241, ``admittance_from_absorption`` :76-87). The coefficient builders
produce the layout the CUDA sweeps read instead of the reference's sparse index list:

* ``wall_shell`` -- for each of the six faces, the pair ``(1/(1+a), a/(1+a))`` for every cell
  on that face, where ``a`` sums ``c dt xi / (2 dx)`` over all absorbing faces touching the
  cell in FACES order, exactly the sum ``wall_update_coefficients`` forms with ``np.add.at``
  (``boundaries.py:167-207``).
* ``layer_profiles`` -- the per-axis ``exp(-sigma dt)`` factors at cell centres and at faces
  (``boundaries.py:244-283``).

Both accept the reference's own objects as well as the ones defined here.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = [
    "FACES",
    "AbsorbingLayer",
    "WallAdmittances",
    "admittance_from_absorption",
    "reflection_coefficient",
    "layer_profiles",
    "wall_shell",
    "wall_cell_coefficients",
    "WallPatches",
    "patch_index",
]

#: Face order used everywhere: (axis, side), side 0 = low, 1 = high (``boundaries.py:73``).
FACES = ((0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1))


def admittance_from_absorption(absorption: float) -> float:
    """Normalised admittance xi = (1 - R)/(1 + R) with R = sqrt(1 - alpha) (``boundaries.py:76-87``)."""
    if not 0.0 <= absorption <= 1.0:
        raise ValueError(f"absorption must be in [0, 1], got {absorption}")
    reflection = math.sqrt(1.0 - absorption)
    return (1.0 - reflection) / (1.0 + reflection)


def reflection_coefficient(normalised_admittance: float, angle: float = 0.0) -> float:
    """Plane-wave pressure reflection (cos t - xi)/(cos t + xi) (``boundaries.py:90-94``)."""
    cosine = math.cos(angle)
    return (cosine - normalised_admittance) / (cosine + normalised_admittance)


@dataclass(frozen=True)
class WallAdmittances:
    """Normalised admittance of each wall, 0 = rigid, 1 = impedance matched."""

    x_min: float = 0.0
    x_max: float = 0.0
    y_min: float = 0.0
    y_max: float = 0.0
    z_min: float = 0.0
    z_max: float = 0.0

    def __post_init__(self) -> None:
        for face, value in zip(FACES, self.values, strict=True):
            if value < 0.0:
                raise ValueError(
                    f"wall {face} has negative admittance {value}: that is a wall that "
                    "generates sound, and it will make the run diverge"
                )

    @property
    def values(self) -> tuple[float, ...]:
        return (self.x_min, self.x_max, self.y_min, self.y_max, self.z_min, self.z_max)

    @property
    def is_rigid(self) -> bool:
        return all(v == 0.0 for v in self.values)

    @classmethod
    def uniform(cls, normalised_admittance: float) -> WallAdmittances:
        return cls(*([normalised_admittance] * 6))

    @classmethod
    def from_absorption(cls, absorption: float) -> WallAdmittances:
        return cls.uniform(admittance_from_absorption(absorption))

    @classmethod
    def matched(cls) -> WallAdmittances:
        return cls.uniform(1.0)


@dataclass(frozen=True)
class AbsorbingLayer:
    """Graded sponge lining the listed faces (``boundaries.py:210-241``)."""

    thickness: int = 16
    target_reflection: float = 1e-5
    order: float = 3.0
    faces: tuple[tuple[int, int], ...] = FACES

    def __post_init__(self) -> None:
        if self.thickness < 1:
            raise ValueError(f"thickness must be at least one cell, got {self.thickness}")
        if not 0.0 < self.target_reflection < 1.0:
            raise ValueError(f"target_reflection must be in (0, 1), got {self.target_reflection}")

    def max_damping(self, dx: float, sound_speed: float) -> float:
        depth = self.thickness * dx
        return -(self.order + 1.0) * sound_speed * math.log(self.target_reflection) / (2.0 * depth)


def patch_index(count: int, patches: int) -> np.ndarray:
    """Patch of each of ``count`` cells along one wall axis: floor(i * patches / count)."""
    return (np.arange(count) * patches) // count


class WallPatches:
    """Per-patch admittances: each wall split into ``patches x patches`` rectangles.

    ``values`` has shape (6, patches, patches) in FACES order, each wall's patches indexed over
    its two other axes in increasing order. A room whose patches on a wall are all equal is the
    reference's ``WallAdmittances`` with that value. The reference has no per-patch walls
    (its ``WallAdmittances`` holds six scalars, ``boundaries.py:120-146``).
    """

    def __init__(self, values) -> None:
        values = np.asarray(values, dtype=np.float64)
        if values.ndim != 3 or values.shape[0] != 6 or values.shape[1] != values.shape[2]:
            raise ValueError(f"values must have shape (6, P, P), got {values.shape}")
        if np.any(values < 0.0):
            raise ValueError("negative admittance: that is a wall that generates sound")
        self.patch_values = values

    @property
    def patches(self) -> int:
        return self.patch_values.shape[1]

    @property
    def values(self) -> tuple[float, ...]:
        """Mean admittance per wall (for code that wants six numbers)."""
        return tuple(float(v.mean()) for v in self.patch_values)

    def face_maps(self, shape) -> list[np.ndarray]:
        maps = []
        for f, (axis, _) in enumerate(FACES):
            b, c = [a for a in range(3) if a != axis]
            ib = patch_index(shape[b], self.patches)
            ic = patch_index(shape[c], self.patches)
            maps.append(self.patch_values[f][np.ix_(ib, ic)])
        return maps

    @classmethod
    def uniform(cls, walls, patches: int) -> WallPatches:
        return cls(np.repeat(np.asarray(walls.values, float)[:, None, None], patches, 1).repeat(patches, 2))


def _face_maps(walls, shape) -> list[np.ndarray]:
    """Admittance of each face as a 2D map over its own (b, c) axes.

    ``walls`` is either a ``WallAdmittances``-like object (six scalars in ``values``) or any
    object with a ``face_maps(shape)`` method returning six 2D arrays (per-patch walls).
    """
    if hasattr(walls, "face_maps"):
        maps = [np.asarray(m, dtype=np.float64) for m in walls.face_maps(shape)]
    else:
        maps = []
        for (axis, _), value in zip(FACES, walls.values, strict=True):
            b, c = [a for a in range(3) if a != axis]
            maps.append(np.full((shape[b], shape[c]), float(value)))
    return maps


def wall_cell_coefficients(shape, sound_speed: float, dt: float, dx: float, walls,
                           force: bool = False):
    """Per-face maps of the summed wall coefficient ``a`` for the cells on each face.

    ``a`` at a cell is the sum, in FACES order, of ``scale * xi_f`` over the faces f that touch
    the cell and have ``xi_f != 0``, with ``scale = c dt / (2 dx)`` -- the reference builds the
    same sum with ``np.add.at`` over its concatenated per-face index lists
    (``boundaries.py:177-207``), which accumulates a cell's faces in FACES order starting from 0.
    Returns six arrays; entry (b, c) of array f belongs to the cell on face f at those
    coordinates. ``None`` when every wall is rigid.
    """
    maps = _face_maps(walls, shape)
    if not force and all(not np.any(m != 0.0) for m in maps):
        return None
    scale = sound_speed * dt / (2.0 * dx)
    n = shape
    out = []
    for axis, side in FACES:
        b, c = [a for a in range(3) if a != axis]
        coords = [None, None, None]
        coords[axis] = np.full((n[b], n[c]), 0 if side == 0 else n[axis] - 1)
        coords[b], coords[c] = np.meshgrid(np.arange(n[b]), np.arange(n[c]), indexing="ij")
        total = np.zeros((n[b], n[c]))
        for (g_axis, g_side), xi_map in zip(FACES, maps, strict=True):
            on_face = coords[g_axis] == (0 if g_side == 0 else n[g_axis] - 1)
            gb, gc = [a for a in range(3) if a != g_axis]
            xi = xi_map[coords[gb], coords[gc]]
            contribution = np.where(on_face & (xi != 0.0), scale * xi, 0.0)
            total = total + contribution
        out.append(total)
    return out


def wall_shell(shape, sound_speed: float, dt: float, dx: float, walls, force: bool = False):
    """Six interleaved ``(1/(1+a), a/(1+a))`` arrays in FP64, or ``None`` when all rigid.

    The two factors are formed from ``a`` in FP64 exactly as ``scheme.py:156-157`` does before
    casting to the working precision. ``force`` returns the shells even for rigid walls (pairs
    (1, 0), which leave the update unchanged), for solvers whose walls will be differentiated.
    """
    sums = wall_cell_coefficients(shape, sound_speed, dt, dx, walls, force)
    if sums is None:
        return None
    shells = []
    for a in sums:
        pair = np.empty(a.shape + (2,))
        pair[..., 0] = 1.0 / (1.0 + a)
        pair[..., 1] = a / (1.0 + a)
        shells.append(np.ascontiguousarray(pair.reshape(-1)))
    return shells


def layer_profiles(shape, dx: float, sound_speed: float, dt: float, layer):
    """``(cell, face)`` damping profiles per axis, FP64 (``boundaries.py:244-283``).

    ``cell[a]`` is sampled at the n_a cell centres, ``face[a]`` at the n_a + 1 faces. A field
    is damped by the profile of its own position on each axis: pressure by ``cell`` on every
    axis, velocity component a by ``face[a]`` on its own axis and ``cell`` on the others.
    """
    thickness = layer.thickness
    order = layer.order
    faces = tuple(tuple(f) for f in layer.faces)
    depth = thickness * dx
    sigma_max = -(order + 1.0) * sound_speed * math.log(layer.target_reflection) / (2.0 * depth)

    def profile(positions: np.ndarray, extent: float, axis: int) -> np.ndarray:
        distance = np.full(positions.shape, np.inf)
        if (axis, 0) in faces:
            distance = np.minimum(distance, positions)
        if (axis, 1) in faces:
            distance = np.minimum(distance, extent - positions)
        inside = np.clip(1.0 - distance / depth, 0.0, 1.0)
        return np.exp(-sigma_max * inside**order * dt)

    cell, face = [], []
    for axis in range(3):
        count = shape[axis]
        extent = count * dx
        cell.append(np.ascontiguousarray(profile((np.arange(count) + 0.5) * dx, extent, axis)))
        face.append(np.ascontiguousarray(profile(np.arange(count + 1) * dx, extent, axis)))
    return cell, face
