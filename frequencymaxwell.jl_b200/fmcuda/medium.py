"""Medium container and phantom generators (mirror of src/medium/types.jl and phantoms.jl).

Every generator describes its phantom as a list of shapes (spheres, plates, cylinders, painted in order over the
background).  With ``on_device=False`` (the reference's behaviour) the shapes are painted into a host array and a
``Medium`` is returned; with ``on_device=True`` a ``DevicePhantom`` is returned, which a solve paints straight
into device memory (fm_phantom_fill) with the same rules, bit for bit, so no permittivity array crosses from the
host.  (The device painting is new; the reference generates on the host.)
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np


class AbstractMedium:
    pass


class Medium(AbstractMedium):
    """Medium(permittivity, permittivity_bg) (medium/types.jl:160-183)."""

    def __init__(self, permittivity: np.ndarray, permittivity_bg: float):
        if not permittivity_bg > 0:
            raise ValueError(f"permittivity_bg must be positive, got: {permittivity_bg}")
        perm = np.asarray(permittivity)
        if perm.ndim != 3:
            raise ValueError("permittivity must be a 3-D array")
        self.permittivity = np.asfortranarray(perm.astype(np.complex128))
        self.permittivity_bg = float(permittivity_bg)

    def __repr__(self):
        g = self.permittivity.shape
        return f"Medium(grid_size={g}, permittivity_bg={self.permittivity_bg})"


SPHERE, PLATE, CYLINDER = 0, 1, 2  # fm_shape kinds (FM_SHAPE_* in include/fmcuda.h)


@dataclass(frozen=True)
class Shape:
    """One painted region: a sphere (centre, radius), a plate (axis = normal 1..3, centre along it, extent =
    thickness) or a cylinder (axis 1..3, centre, radius, extent = height).  Centres are 1-based voxel
    coordinates."""
    kind: int
    center: Tuple[float, float, float]
    value: complex
    radius: float = 0.0
    axis: int = 3
    extent: float = 0.0


class DevicePhantom(AbstractMedium):
    """A phantom given by its shapes, painted on the device when a solve builds its potential.

    ``permittivity`` paints the same shapes on the host (for inspection, or for paths that need the array)."""

    def __init__(self, grid_size: Sequence[int], shapes: Sequence[Shape], permittivity_bg: float):
        if not permittivity_bg > 0:
            raise ValueError(f"permittivity_bg must be positive, got: {permittivity_bg}")
        self.grid_size = tuple(int(n) for n in grid_size)
        self.shapes: List[Shape] = list(shapes)
        self.permittivity_bg = float(permittivity_bg)

    @property
    def permittivity(self) -> np.ndarray:
        return paint_host(self.grid_size, self.shapes, self.permittivity_bg)

    def __repr__(self):
        return f"DevicePhantom(grid_size={self.grid_size}, shapes={len(self.shapes)}, permittivity_bg={self.permittivity_bg})"


def permittivity(m: AbstractMedium) -> np.ndarray:
    return m.permittivity


def permittivity_bg(m: AbstractMedium) -> float:
    return m.permittivity_bg


def grid_size(m: AbstractMedium) -> Tuple[int, int, int]:
    if isinstance(m, DevicePhantom):
        return m.grid_size
    return tuple(m.permittivity.shape)


def _round_int(x: float) -> int:
    return int(round(x))


def fill_sphere(ph: np.ndarray, center, radius: float, value: complex) -> None:
    """_fill_sphere! (phantoms.jl:212-247): 1-based centre, bounding box by round, <= r^2."""
    g = ph.shape
    lo = [max(1, _round_int(center[d] - radius)) for d in range(3)]
    hi = [min(g[d], _round_int(center[d] + radius)) for d in range(3)]
    if any(hi[d] < lo[d] for d in range(3)):
        return
    i = np.arange(lo[0], hi[0] + 1).reshape(-1, 1, 1) - center[0]
    j = np.arange(lo[1], hi[1] + 1).reshape(1, -1, 1) - center[1]
    k = np.arange(lo[2], hi[2] + 1).reshape(1, 1, -1) - center[2]
    mask = i * i + j * j + k * k <= radius ** 2
    sub = ph[lo[0] - 1:hi[0], lo[1] - 1:hi[1], lo[2] - 1:hi[2]]
    sub[mask] = value


def _fill_plate(ph: np.ndarray, axis: int, center: float, thickness: float, value: complex) -> None:
    """phantom_plate's slab (phantoms.jl:184-196): [max(1, round(c - t/2)), min(N, round(c + t/2))] along the normal."""
    n = ph.shape[axis - 1]
    s = max(1, _round_int(center - thickness / 2))
    e = min(n, _round_int(center + thickness / 2))
    sl = [slice(None)] * 3
    sl[axis - 1] = slice(s - 1, e)
    ph[tuple(sl)] = value


def _fill_cylinder(ph: np.ndarray, axis: int, center, radius: float, height: float, value: complex) -> None:
    """phantom_cylinder / _fill_cylinder! (phantoms.jl:299-362): the axis range as for a plate, and the squared
    distance over the two other axes (increasing axis order) <= r^2."""
    g = ph.shape
    a = axis - 1
    s = max(1, _round_int(center[a] - height / 2))
    e = min(g[a], _round_int(center[a] + height / 2))
    others = [d for d in range(3) if d != a]
    u = (np.arange(1, g[others[0]] + 1) - center[others[0]]).reshape(-1, 1)
    v = (np.arange(1, g[others[1]] + 1) - center[others[1]]).reshape(1, -1)
    disk = u * u + v * v <= radius ** 2
    for idx in range(s - 1, e):
        sl = [slice(None)] * 3
        sl[a] = idx
        plane = ph[tuple(sl)]
        plane[disk] = value


def paint_host(grid_size: Sequence[int], shapes: Sequence[Shape], permittivity_bg: float) -> np.ndarray:
    """The background, then every shape in order (later shapes overwrite earlier ones), as the reference's
    generators fill their array."""
    g = tuple(int(n) for n in grid_size)
    ph = np.full(g, complex(permittivity_bg), dtype=np.complex128, order="F")
    for sh in shapes:
        if sh.kind == SPHERE:
            fill_sphere(ph, sh.center, sh.radius, complex(sh.value))
        elif sh.kind == PLATE:
            _fill_plate(ph, sh.axis, sh.center[sh.axis - 1], sh.extent, complex(sh.value))
        elif sh.kind == CYLINDER:
            _fill_cylinder(ph, sh.axis, sh.center, sh.radius, sh.extent, complex(sh.value))
        else:
            raise ValueError(f"unknown shape kind {sh.kind}")
    return ph


def _medium(grid_size, shapes, permittivity_bg, on_device: bool) -> AbstractMedium:
    if on_device:
        return DevicePhantom(grid_size, shapes, permittivity_bg)
    return Medium(paint_host(grid_size, shapes, permittivity_bg), permittivity_bg)


def phantom_bead(grid_size: Sequence[int], permittivity_profile: Sequence[complex], pixel_radius: float,
                 permittivity_bg: float = 1.0, bead_distance: Optional[float] = None,
                 on_device: bool = False) -> AbstractMedium:
    """phantom_bead (phantoms.jl:58-106)."""
    if bead_distance is None:
        bead_distance = 2 * pixel_radius
    if not all(n > 0 for n in grid_size):
        raise ValueError("grid_size must have positive dimensions")
    if not pixel_radius > 0:
        raise ValueError("pixel_radius must be positive")
    if len(permittivity_profile) == 0:
        raise ValueError("permittivity_profile cannot be empty")
    if not permittivity_bg > 0:
        raise ValueError("permittivity_bg must be positive")
    g = tuple(int(n) for n in grid_size)
    num = len(permittivity_profile)
    c = [(g[d] + 1) / 2 for d in range(3)]
    shapes = []
    for b in range(1, num + 1):
        zc = c[2] + (b - (num + 1) / 2) * bead_distance
        if zc < 1 or zc > g[2]:
            continue
        shapes.append(Shape(SPHERE, (c[0], c[1], zc), complex(permittivity_profile[(b - 1) % num]),
                            radius=pixel_radius))
    return _medium(g, shapes, permittivity_bg, on_device)


def phantom_plate(grid_size: Sequence[int], permittivity_profile: Sequence[complex], thickness_pixel: float,
                  permittivity_bg: float = 1.0, plate_normal: int = 3, on_device: bool = False) -> AbstractMedium:
    """phantom_plate (phantoms.jl:156-199)."""
    if not all(n > 0 for n in grid_size):
        raise ValueError("grid_size must have positive dimensions")
    if not thickness_pixel > 0:
        raise ValueError("thickness_pixel must be positive")
    if not 1 <= plate_normal <= 3:
        raise ValueError("plate_normal must be 1, 2, or 3")
    if len(permittivity_profile) == 0:
        raise ValueError("permittivity_profile cannot be empty")
    if not permittivity_bg > 0:
        raise ValueError("permittivity_bg must be positive")
    g = tuple(int(n) for n in grid_size)
    c = tuple((g[d] + 1) / 2 for d in range(3))
    shapes = [Shape(PLATE, c, complex(permittivity_profile[0]), axis=plate_normal, extent=thickness_pixel)]
    return _medium(g, shapes, permittivity_bg, on_device)


def phantom_cylinder(grid_size: Sequence[int], permittivity_profile: Sequence[complex], radius_pixel: float,
                     permittivity_bg: float = 1.0, height_pixel: Optional[float] = None, axis: int = 3,
                     on_device: bool = False) -> AbstractMedium:
    """phantom_cylinder (phantoms.jl:272-362)."""
    if height_pixel is None:
        height_pixel = 2 * radius_pixel
    if not all(n > 0 for n in grid_size):
        raise ValueError("grid_size must have positive dimensions")
    if not radius_pixel > 0 or not height_pixel > 0:
        raise ValueError("radius_pixel and height_pixel must be positive")
    if not 1 <= axis <= 3:
        raise ValueError("axis must be 1, 2, or 3")
    if len(permittivity_profile) == 0:
        raise ValueError("permittivity_profile cannot be empty")
    if not permittivity_bg > 0:
        raise ValueError("permittivity_bg must be positive")
    g = tuple(int(n) for n in grid_size)
    c = tuple((g[d] + 1) / 2 for d in range(3))
    shapes = [Shape(CYLINDER, c, complex(permittivity_profile[0]), radius=radius_pixel, axis=axis,
                    extent=height_pixel)]
    return _medium(g, shapes, permittivity_bg, on_device)


def phantom_random_beads(grid_size: Sequence[int], count: int, radius_range: Tuple[float, float],
                         index_range: Tuple[float, float], permittivity_bg: float, seed: int,
                         max_tries: int = 200000, on_device: bool = False) -> AbstractMedium:
    """Seeded phantom of non-overlapping beads (new; not in the reference).

    Radii ~ U[radius_range] px, refractive indices ~ U[index_range] (permittivity n^2), centres drawn
    uniformly with the whole bead inside the grid and centre distance >= r1 + r2 + 1 to every earlier
    bead (rejection sampling).  Beads are drawn with the reference's sphere rule (fill_sphere)."""
    rng = np.random.default_rng(seed)
    g = tuple(int(n) for n in grid_size)
    placed = []
    tries = 0
    while len(placed) < count:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place all beads")
        r = rng.uniform(*radius_range)
        n = rng.uniform(*index_range)
        lo = [1 + r for _ in range(3)]
        hi = [g[d] - r for d in range(3)]
        if any(hi[d] < lo[d] for d in range(3)):
            continue
        ctr = [rng.uniform(lo[d], hi[d]) for d in range(3)]
        if all(np.linalg.norm(np.subtract(ctr, p[0])) >= r + p[1] + 1 for p in placed):
            placed.append((ctr, r, n))
    shapes = [Shape(SPHERE, tuple(ctr), complex(n * n), radius=r) for ctr, r, n in placed]
    return _medium(g, shapes, permittivity_bg, on_device)
