"""Plane-wave sources (mirror of src/sources/plane_wave.jl and field_generation.jl)."""
from __future__ import annotations

import math
from typing import List, Sequence, Union

import numpy as np

from .boundary import padding_pixels


class AbstractCurrentSource:
    pass


class PlaneWaveSource(AbstractCurrentSource):
    """PlaneWaveSource(wavelength, polarization, k_vector, amplitude=1, phase=0) with the
    reference's validation (plane_wave.jl:63-116): |k| = 1 and real(pol . k) = 0 to 1e-10."""

    def __init__(self, wavelength: float, polarization: Sequence[complex], k_vector: Sequence[float],
                 amplitude: float = 1.0, phase: float = 0.0):
        self.wavelength = float(wavelength)
        self.polarization = np.asarray(polarization, dtype=np.complex128).reshape(3)
        self.k_vector = np.asarray(k_vector, dtype=np.float64).reshape(3)
        self.amplitude = float(amplitude)
        self.phase = float(phase)
        if not self.wavelength > 0:
            raise ValueError("wavelength must be positive")
        if not self.amplitude >= 0:
            raise ValueError("amplitude must be non-negative")
        if not abs(np.linalg.norm(self.k_vector) - 1) < 1e-10:
            raise ValueError("k_vector must be normalized (|k| = 1)")
        if not abs(np.real(np.vdot(self.polarization, self.k_vector))) < 1e-10:
            raise ValueError("polarization must be transverse to k_vector")

    def __repr__(self):
        return (f"PlaneWaveSource(wavelength={self.wavelength}, polarization={self.polarization.tolist()}, "
                f"k_vector={self.k_vector.tolist()}, amplitude={self.amplitude}, phase={self.phase})")


Sources = Union[PlaneWaveSource, Sequence[PlaneWaveSource]]


def source_wavelength(sources: Sources) -> float:
    """plane_wave.jl:125-141."""
    if isinstance(sources, PlaneWaveSource):
        return sources.wavelength
    w = sources[0].wavelength
    for s in sources[1:]:
        if s.wavelength != w:
            raise ValueError("All sources must have the same wavelength for coherent superposition")
    return w


def as_list(sources: Sources):
    if isinstance(sources, PlaneWaveSource):
        return [sources]
    sources = list(sources)
    if len(sources) == 0:
        raise ValueError("sources vector cannot be empty")
    w0 = sources[0].wavelength
    for s in sources[1:]:
        if not math.isclose(s.wavelength, w0, rel_tol=1e-10):
            raise ValueError("All sources must have the same wavelength for coherent interference.")
    return sources


def polarisation_vectors(src: PlaneWaveSource, permittivity_bg: float):
    """E_perp, H_perp and the in-medium k vector (plane_wave.jl:218-232)."""
    k_bg = 2 * math.pi / src.wavelength * math.sqrt(permittivity_bg)
    k_hat = src.k_vector / np.linalg.norm(src.k_vector)
    E0 = src.polarization / np.linalg.norm(src.polarization)
    E_perp = E0 - np.vdot(E0, k_hat) * k_hat
    E_perp = E_perp / np.linalg.norm(E_perp)
    H_perp = np.cross(k_hat, E_perp) / (377 / math.sqrt(permittivity_bg))
    return E_perp, H_perp, k_bg * k_hat


def generate_incident_field(sources: Sources, solver, permittivity_bg: float = 1.0):
    """Incident E, H on the solver's padded grid (plane_wave.jl:198-268, field_generation.jl:42-78).

    Host-side and vectorised; the device solve evaluates the same fields itself."""
    from .fields import ElectromagneticField
    srcs = as_list(sources)
    g, res = solver.grid_size, solver.resolution
    pad = [padding_pixels(solver.boundary_conditions[d], res[d]) for d in range(3)]
    P = tuple(g[d] + 2 * pad[d] for d in range(3))
    E = np.zeros(P + (3,), dtype=np.complex128, order="F")
    H = np.zeros(P + (3,), dtype=np.complex128, order="F")
    center = [(g[d] - 1) * res[d] / 2 for d in range(3)]
    for src in srcs:
        Ep, Hp, kv = polarisation_vectors(src, permittivity_bg)
        r = [(np.arange(P[d]) - pad[d]) * res[d] - center[d] for d in range(3)]
        ph = (kv[0] * r[0]).reshape(-1, 1, 1) + (kv[1] * r[1]).reshape(1, -1, 1) + \
            (kv[2] * r[2]).reshape(1, 1, -1) + src.phase
        amp = src.amplitude * np.exp(1j * ph)
        for c in range(3):
            E[..., c] += amp * Ep[c]
            H[..., c] += amp * Hp[c]
    return ElectromagneticField(E, H, res, srcs[0].wavelength)


def illumination_cone(grid_size, resolution, wavelength: float, permittivity_bg: float, n_angles: int, na: float,
                      seed: int, polarizations: str = "sp") -> List[PlaneWaveSource]:
    """Seeded illumination set (new; not in the reference): ``n_angles`` directions with (kx, ky) uniform in
    the disk sin(theta) <= NA / n_bg, snapped to the lattice 2*pi*m/(N*dx) of the grid's x and y axes, each
    with the polarisations named in ``polarizations`` ("s": k x z normalised, "p": s x k), both transverse
    to k.  Returns the sources angle-major (s then p per angle)."""
    rng = np.random.default_rng(seed + 1)
    nbg = math.sqrt(permittivity_bg)
    kbg = 2 * math.pi * nbg / wavelength
    dk = [2 * math.pi / (grid_size[d] * resolution[d]) for d in range(2)]
    ks = []
    while len(ks) < n_angles:
        r = math.sqrt(rng.uniform()) * na / nbg
        phi = rng.uniform(0, 2 * math.pi)
        kx, ky = kbg * r * math.cos(phi), kbg * r * math.sin(phi)
        kx = round(kx / dk[0]) * dk[0]
        ky = round(ky / dk[1]) * dk[1]
        st = math.hypot(kx, ky) / kbg
        if st > na / nbg:
            continue
        k = np.array([kx / kbg, ky / kbg, math.sqrt(max(0.0, 1 - st * st))])
        ks.append(k / np.linalg.norm(k))
    out = []
    for k in ks:
        s = np.cross(k, [0.0, 0.0, 1.0])
        if np.linalg.norm(s) < 1e-12:
            s = np.array([0.0, 1.0, 0.0])
        s /= np.linalg.norm(s)
        p = np.cross(s, k)
        p /= np.linalg.norm(p)
        for c in polarizations:
            out.append(PlaneWaveSource(wavelength=wavelength, polarization=s if c == "s" else p, k_vector=k))
    return out
