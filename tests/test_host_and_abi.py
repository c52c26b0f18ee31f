"""Host-side mirror of the reference API (no GPU needed) and the C-ABI library surface."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import cbs_oracle as O

import fmcuda as F
from fmcuda import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "fmcuda.h")).read()
    return set(re.findall(r"^\s*(?:fm_status|int|void|long long|const char\*|void\*)\s+(fm_\w+)\(", txt, re.M))


def test_library_exports_every_header_symbol():
    assert os.path.exists(_lib.LIB_PATH), "build libfmcuda.so first"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = _header_functions()
    assert declared, "no declarations parsed"
    assert declared <= exported, declared - exported
    assert set(_lib.EXPORTED) == declared


def _header_constants():
    """FM_* enumerators and defines of include/fmcuda.h with their values."""
    txt = open(os.path.join(ROOT, "include", "fmcuda.h")).read()
    vals = {}
    for body in re.findall(r"enum\s*\{([^}]*)\}", txt):
        for name, v in re.findall(r"(FM_\w+)\s*=\s*(-?\d+)", body):
            vals[name] = int(v)
    return vals


def test_binding_constants_match_the_header():
    """The ctypes mirror and the Julia binding use the header's values for every constant they name."""
    hdr = _header_constants()
    assert {"FM_ORTHO_BLOCK", "FM_BLOCK_FP64_ORTHO", "FM_TUNE_BLOCK_DOT", "FM_PREC_F32_MATH64"} <= set(hdr)
    py = {k: getattr(_lib, k) for k in dir(_lib) if k.startswith("FM_") and isinstance(getattr(_lib, k), int)}
    for k, v in py.items():
        if k in hdr:
            assert hdr[k] == v, (k, v, hdr[k])
    jl = open(os.path.join(ROOT, "frequencymaxwell.jl_b200", "julia", "FrequencyMaxwellCUDA.jl")).read()
    named = dict((k, int(v)) for k, v in re.findall(r"const (FM_\w+) = Cint\((-?\d+)\)", jl))
    assert len(named) >= 10
    for k, v in named.items():
        assert hdr.get(k) == v, (k, v, hdr.get(k))


def test_library_loads_without_gpu_calls():
    L = _lib.lib()
    assert L.fm_abi_version() == 2
    assert isinstance(L.fm_device_count(), int)
    assert L.fm_last_error() is not None


def test_plan_rejects_bad_descriptions():
    L = _lib.lib()
    d = _lib.fm_plan_desc()
    h = ctypes.c_void_p()
    d.grid[:] = [0, 8, 8]
    d.resolution[:] = [1, 1, 1]
    d.precision = 1
    assert L.fm_plan_create(ctypes.byref(d), ctypes.byref(h)) != 0
    assert not h


def test_boundary_mirror_matches_oracle():
    for prof_o, prof_f in [(O.TANH, F.TanhProfile), (O.EXPONENTIAL, F.ExponentialProfile),
                           (O.TUKEY, F.TukeyProfile)]:
        for L in (0, 1, 5, 32):
            np.testing.assert_array_equal(F.create_attenuation_window(prof_f, L), O.attenuation_window(prof_o, L))
    bo = O.AbsorbingBC(1.5e-6, 1.0e-6, 0.8, O.TUKEY)
    bf = F.AbsorbingBoundaryCondition(thickness=1.5e-6, attenuation_thickness=1.0e-6, sharpness=0.8,
                                      profile=F.TukeyProfile)
    cfg = O.SolverConfig((50e-9,) * 3, (16, 16, 20), (O.PeriodicBC(), O.PeriodicBC(), bo))
    fo = O.attenuation_filters(cfg)[2]
    ff = F.attenuation_filter(bf, 50e-9, 20)
    np.testing.assert_array_equal(ff, fo)
    assert F.padding_pixels(bf, 50e-9) == O.padding_pixels(bo, 50e-9)
    with pytest.raises(ValueError):
        F.AbsorbingBoundaryCondition(thickness=1e-6, attenuation_thickness=2e-6)


def test_phantoms_match_oracle():
    for g, eps, r in [((32, 32, 32), [2.25], 8), ((21, 22, 23), [2.0, 3.0], 4.5), ((20, 20, 20), [2.0], 15)]:
        np.testing.assert_array_equal(F.phantom_bead(g, eps, r, permittivity_bg=1.7).permittivity,
                                      O.phantom_bead(g, eps, r, permittivity_bg=1.7))
    np.testing.assert_array_equal(F.phantom_plate((21, 50, 50), [2.0], 4, permittivity_bg=1.0).permittivity,
                                  O.phantom_plate((21, 50, 50), [2.0], 4, permittivity_bg=1.0))
    for ax in (1, 2, 3):
        np.testing.assert_array_equal(
            F.phantom_cylinder((21, 30, 17), [2.0 + 0.1j], 5.5, permittivity_bg=1.3, height_pixel=7, axis=ax).permittivity,
            O.phantom_cylinder((21, 30, 17), [2.0 + 0.1j], 5.5, permittivity_bg=1.3, height_pixel=7, axis=ax))
    m = F.phantom_random_beads((64, 64, 32), 6, (2, 6), (1.36, 1.6), 1.33 ** 2, 3)
    assert m.permittivity.shape == (64, 64, 32)
    assert np.all(m.permittivity.real >= 1.33 ** 2 - 1e-12)


def test_device_phantom_shapes_paint_like_the_host_generators():
    """on_device=True returns the shape list; painting it on the host gives the generator's array."""
    cases = [lambda d: F.phantom_bead((21, 22, 23), [2.0, 3.0], 4.5, permittivity_bg=1.7, on_device=d),
             lambda d: F.phantom_plate((21, 50, 50), [2.0], 4, permittivity_bg=1.0, plate_normal=2, on_device=d),
             lambda d: F.phantom_cylinder((21, 30, 17), [2.0], 5.5, permittivity_bg=1.3, axis=1, on_device=d),
             lambda d: F.phantom_random_beads((64, 64, 32), 6, (2, 6), (1.36, 1.6), 1.33 ** 2, 3, on_device=d)]
    for make in cases:
        host, dev = make(False), make(True)
        assert isinstance(dev, F.DevicePhantom) and F.grid_size(dev) == host.permittivity.shape
        np.testing.assert_array_equal(dev.permittivity, host.permittivity)
    # later shapes overwrite earlier ones; bounding boxes round half to even (round(2.5) = 2)
    sh = [F.Shape(0, (4.5, 4.5, 4.5), 2.0, radius=2.0), F.Shape(1, (0, 0, 4.5), 3.0, axis=3, extent=1.0),
          F.Shape(2, (4.5, 4.5, 4.5), 4.0, radius=1.0, axis=1, extent=3.0)]
    ph = F.paint_host((8, 8, 8), sh, 1.0)
    assert ph[3, 3, 3] == 4.0 and ph[0, 0, 3] == 3.0 and ph[0, 0, 4] == 3.0 and ph[0, 0, 5] == 1.0


def test_incident_field_matches_oracle():
    bz = F.AbsorbingBoundaryCondition(thickness=0.8e-6, attenuation_thickness=0.8e-6, sharpness=1.0)
    solver = F.ConvergentBornSolver(resolution=(50e-9,) * 3, grid_size=(16, 16, 16),
                                    boundary_conditions=(F.PeriodicBoundaryCondition(),) * 2 + (bz,))
    cfg = O.SolverConfig((50e-9,) * 3, (16, 16, 16), (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(0.8e-6, 0.8e-6, 1.0)))
    k = np.array([0.3, 0.2, np.sqrt(1 - 0.13)])
    srcs_f = [F.PlaneWaveSource(wavelength=500e-9, polarization=[0, 1, -0.2 / np.sqrt(0.87)], k_vector=k, phase=0.3),
              F.PlaneWaveSource(wavelength=500e-9, polarization=[1, 1j, 0], k_vector=[0, 0, 1], amplitude=2.0)]
    srcs_o = [O.PlaneWave(500e-9, s.polarization, s.k_vector, s.amplitude, s.phase) for s in srcs_f]
    f = F.generate_incident_field(srcs_f, solver, permittivity_bg=1.7)
    Eo, Ho = O.incident_field(srcs_o, cfg, 1.7)
    assert O.rel_l2(f.E, Eo) < 1e-13 and O.rel_l2(f.H, Ho) < 1e-13


def test_solver_mirror_validation():
    with pytest.raises(ValueError):
        F.ConvergentBornSolver(resolution=(50e-9,) * 3, grid_size=(8, 8, 8),
                               boundary_conditions=F.PeriodicBoundaryCondition(), tolerance=1.5)
    with pytest.raises(ValueError):
        F.ConvergentBornSolver(resolution=(50e-9,) * 3, grid_size=(8, 8, 8),
                               boundary_conditions=F.PeriodicBoundaryCondition(), device="cpu")
    bz = F.AbsorbingBoundaryCondition(thickness=1e-6, attenuation_thickness=1e-6)
    s = F.ConvergentBornSolver(resolution=(50e-9,) * 3, grid_size=(32, 32, 16),
                               boundary_conditions=(F.PeriodicBoundaryCondition(),) * 2 + (bz,))
    assert s.compute_ROI() == (1, 32, 1, 32, 11, 26)
    assert F.domain_size(s) == pytest.approx((32 * 50e-9, 32 * 50e-9, 16 * 50e-9))
    o = s.solve_options(16)
    assert o.maxiters == 100 and o.reltol == 1e-6 and o.abstol == pytest.approx(1e-8)
    assert s.solve_options(60).maxiters == 120
    F.reset(s)
    assert s.iteration_count == 0 and s.residual_history == []


def test_sources_validation():
    with pytest.raises(ValueError):
        F.PlaneWaveSource(wavelength=500e-9, polarization=[0, 0, 1], k_vector=[0, 0, 1])
    with pytest.raises(ValueError):
        F.source_wavelength([F.PlaneWaveSource(wavelength=500e-9, polarization=[1, 0, 0], k_vector=[0, 0, 1]),
                             F.PlaneWaveSource(wavelength=501e-9, polarization=[1, 0, 0], k_vector=[0, 0, 1])])
