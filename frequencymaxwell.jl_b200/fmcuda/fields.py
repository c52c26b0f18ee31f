"""Field container (mirror of src/fields/electromagnetic_field.jl)."""
from __future__ import annotations

import math

import numpy as np


class ElectromagneticField:
    """ElectromagneticField(E, H, resolution, wavelength) (electromagnetic_field.jl:46-90)."""

    def __init__(self, E: np.ndarray, H: np.ndarray, resolution, wavelength: float):
        if E.shape != H.shape:
            raise ValueError("Efield and Hfield arrays must have same size")
        if E.ndim == 4 and E.shape[3] != 3:
            raise ValueError("field arrays must have 3 components in last dimension")
        if not all(r > 0 for r in resolution):
            raise ValueError("resolution must be positive")
        if not wavelength > 0:
            raise ValueError("wavelength must be positive")
        self.E = E
        self.H = H
        self.resolution = tuple(float(r) for r in resolution)
        self.wavelength = float(wavelength)

    def __add__(self, other: "ElectromagneticField") -> "ElectromagneticField":
        """electromagnetic_field.jl:252-266."""
        if self.E.shape != other.E.shape:
            raise ValueError(f"Fields must have same grid size: {self.E.shape} vs {other.E.shape}")
        if self.resolution != other.resolution:
            raise ValueError("Fields must have same resolution")
        if not math.isclose(self.wavelength, other.wavelength, rel_tol=1e-10):
            raise ValueError("Fields must have same wavelength")
        return ElectromagneticField(self.E + other.E, self.H + other.H, self.resolution, self.wavelength)

    def __repr__(self):
        return (f"ElectromagneticField(grid_size={self.E.shape}, resolution={self.resolution}, "
                f"wavelength={self.wavelength})")


def domain_size(f: ElectromagneticField):
    g = f.E.shape[:3]
    return tuple(g[i] * f.resolution[i] for i in range(3))


def crop_to_ROI(f: ElectromagneticField, solver) -> ElectromagneticField:
    """electromagnetic_field.jl:288-303."""
    r = solver.compute_ROI()
    sl = (slice(r[0] - 1, r[1]), slice(r[2] - 1, r[3]), slice(r[4] - 1, r[5]), slice(None))
    return ElectromagneticField(np.asfortranarray(f.E[sl]), np.asfortranarray(f.H[sl]), solver.resolution,
                                f.wavelength)


def to_host(f: ElectromagneticField) -> ElectromagneticField:
    """Fields returned by this package are already host arrays (electromagnetic_field.jl:324-333)."""
    return f


def field_energy(f: ElectromagneticField) -> float:
    """electromagnetic_field.jl:112-127."""
    e0, mu0 = 8.854187817e-12, 4 * math.pi * 1e-7
    return (e0 * float(np.sum(np.abs(f.E) ** 2)) + mu0 * float(np.sum(np.abs(f.H) ** 2))) / 2 * \
        float(np.prod(f.resolution))


def field_intensity(f: ElectromagneticField, component: str = "total") -> np.ndarray:
    """electromagnetic_field.jl:171-186."""
    if component == "total":
        return np.sum(np.abs(f.E) ** 2, axis=3)
    idx = {"x": 0, "y": 1, "z": 2}.get(component)
    if idx is None:
        raise ValueError("component must be :total, :x, :y, or :z")
    return np.abs(f.E[..., idx]) ** 2
