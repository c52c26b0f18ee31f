"""fmcuda: the convergent Born series solve of FrequencyMaxwell.jl on NVIDIA B200 (sm_100a).

Python mirror of the reference's public API for the solve path (ConvergentBornSolver,
PlaneWaveSource, Medium, phantoms, solve) driving libfmcuda through its C ABI.
"""
from .boundary import (AbsorbingBoundaryCondition, AbstractBoundaryCondition, AttenuationProfile,
                       ExponentialProfile, PeriodicBoundaryCondition, TanhProfile, TukeyProfile, attenuation_filter,
                       create_attenuation_window, padding_pixels, requires_averaging, requires_padding,
                       subpixel_shift)
from .fields import ElectromagneticField, crop_to_ROI, field_energy, field_intensity, to_host
from .medium import (AbstractMedium, DevicePhantom, Medium, Shape, grid_size, paint_host, permittivity,
                     permittivity_bg, phantom_bead, phantom_cylinder, phantom_plate, phantom_random_beads)
from .solver import (BornSeries, ConvergentBornSolver, DevicePlan, KrylovJL_BICGSTAB, KrylovJL_GMRES, compute_ROI,
                     domain_size, grid_spacing, reset, solve, solve_batch)
from .sources import (AbstractCurrentSource, PlaneWaveSource, generate_incident_field, illumination_cone,
                      source_wavelength)
from . import _lib, autotune as autotuner

__all__ = [n for n in dir() if not n.startswith("_")]
