"""Boundary conditions (mirror of src/solvers/boundary_conditions.jl).

These are host-side parameters of the solve: padding, sub-pixel shift,
averaging flag and the 1-D attenuation windows that the device multiplies into
the potential.
"""
from __future__ import annotations

import enum
import math
from dataclasses import dataclass

import numpy as np


class AttenuationProfile(enum.Enum):
    """boundary_conditions.jl:228-232."""
    TanhProfile = 0
    ExponentialProfile = 1
    TukeyProfile = 2


TanhProfile = AttenuationProfile.TanhProfile
ExponentialProfile = AttenuationProfile.ExponentialProfile
TukeyProfile = AttenuationProfile.TukeyProfile


class AbstractBoundaryCondition:
    pass


@dataclass(frozen=True)
class PeriodicBoundaryCondition(AbstractBoundaryCondition):
    """boundary_conditions.jl:157-181."""

    def __repr__(self):
        return "PeriodicBoundaryCondition()"


@dataclass(frozen=True)
class AbsorbingBoundaryCondition(AbstractBoundaryCondition):
    """boundary_conditions.jl:335-395, with the same validation (ValueError for ArgumentError)."""
    thickness: float
    attenuation_thickness: float
    sharpness: float = 0.9
    profile: AttenuationProfile = TanhProfile

    def __post_init__(self):
        if not self.thickness > 0:
            raise ValueError(f"thickness must be positive, got: {self.thickness}")
        if not self.attenuation_thickness > 0:
            raise ValueError(f"attenuation_thickness must be positive, got: {self.attenuation_thickness}")
        if not self.attenuation_thickness <= self.thickness:
            raise ValueError(f"attenuation_thickness ({self.attenuation_thickness}) must be <= thickness "
                             f"({self.thickness})")
        if not (0 <= self.sharpness <= 1):
            raise ValueError(f"sharpness must be in [0, 1], got: {self.sharpness}")
        if not isinstance(self.profile, AttenuationProfile):
            raise ValueError(f"Unknown attenuation profile: {self.profile}")


def _round_int(x: float) -> int:
    # Julia round(Int, x): nearest, ties to even
    return int(round(x))


def padding_pixels(bc: AbstractBoundaryCondition, resolution: float) -> int:
    """boundary_conditions.jl:450-459."""
    if isinstance(bc, PeriodicBoundaryCondition):
        return 0
    return _round_int(bc.thickness / (resolution * 2))


def subpixel_shift(bc: AbstractBoundaryCondition) -> float:
    """boundary_conditions.jl:518-527."""
    return 0.0 if isinstance(bc, PeriodicBoundaryCondition) else 0.25


def requires_padding(bc: AbstractBoundaryCondition) -> bool:
    """boundary_conditions.jl:567-573."""
    return isinstance(bc, AbsorbingBoundaryCondition)


def requires_averaging(bc: AbstractBoundaryCondition) -> bool:
    """boundary_conditions.jl:609-615."""
    return isinstance(bc, AbsorbingBoundaryCondition)


def create_attenuation_window(profile: AttenuationProfile, L: int) -> np.ndarray:
    """_create_attenuation_window (boundary_conditions.jl:632-658), including the Tanh form's
    operator order (tanh(x)/tanh(2.5) - tanh(-2.5))/2."""
    if L <= 0:
        return np.zeros(0)
    if profile == TanhProfile:
        t = np.tanh(np.linspace(-2.5, 2.5, L))
        return (t / math.tanh(2.5) - math.tanh(-2.5)) / 2
    x = np.linspace(0.0, 1.0, L)
    if profile == ExponentialProfile:
        return np.exp(-(((1.0 - x) / 0.3) ** 2))
    if profile == TukeyProfile:
        return 0.5 * (1.0 + np.cos(np.pi * (1.0 - x)))
    raise ValueError(f"Unknown attenuation profile: {profile}")


def attenuation_filter(bc: AbstractBoundaryCondition, resolution: float, roi_size: int) -> np.ndarray:
    """The 1-D filter that _apply_attenuation_to_potential! multiplies along one axis
    (convergent_born.jl:893-944); all ones where the boundary needs no attenuation."""
    pad = padding_pixels(bc, resolution)
    n = roi_size + 2 * pad
    if not requires_padding(bc) or pad == 0:
        return np.ones(n)
    att = _round_int(bc.attenuation_thickness / (resolution * 2))
    L = min(pad, att)
    w = create_attenuation_window(bc.profile, L)
    w = w * bc.sharpness + (1 - bc.sharpness)
    return np.concatenate([w, np.ones(roi_size + 2 * (pad - L)), w[::-1]])
