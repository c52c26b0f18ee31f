"""Pins of the CPU oracle against the constants that the reference's own tests assert.

Each test restates an assertion of FrequencyMaxwell.jl's test suite (file:line given) and checks the
oracle against it.  These are the only known answers the reference provides for this path: no
reference test calls solve (test/runtests.jl:5-10)."""
import math

import numpy as np
import pytest

from oracle import cbs_oracle as O


def test_padding_pixels():
    # test/solvers/boundary_conditions.jl:80-97
    assert O.padding_pixels(O.PeriodicBC(), 50e-9) == 0
    assert O.padding_pixels(O.PeriodicBC(), 100e-9) == 0
    bc = O.AbsorbingBC(2.0e-6, 1.5e-6)
    assert O.padding_pixels(bc, 50e-9) == round(2.0e-6 / (50e-9 * 2)) == 20
    assert O.padding_pixels(bc, 100e-9) == round(2.0e-6 / (100e-9 * 2)) == 10


def test_shift_padding_averaging_flags():
    # test/solvers/boundary_conditions.jl:99-137
    bc = O.AbsorbingBC(2.0e-6, 1.5e-6)
    assert O.subpixel_shift(O.PeriodicBC()) == 0.0
    assert O.subpixel_shift(bc) == 0.25
    assert O.requires_padding(O.PeriodicBC()) is False and O.requires_padding(bc) is True
    assert O.requires_averaging(O.PeriodicBC()) is False and O.requires_averaging(bc) is True


def test_absorbing_defaults_and_validation():
    # test/solvers/boundary_conditions.jl:20-78
    bc = O.AbsorbingBC(2.0e-6, 1.5e-6)
    assert bc.sharpness == pytest.approx(0.9) and bc.profile == O.TANH
    for kw in [dict(thickness=-1e-6, attenuation_thickness=0.5e-6),
               dict(thickness=2e-6, attenuation_thickness=-0.5e-6),
               dict(thickness=1e-6, attenuation_thickness=2e-6),
               dict(thickness=2e-6, attenuation_thickness=1e-6, sharpness=-0.1),
               dict(thickness=2e-6, attenuation_thickness=1e-6, sharpness=1.5)]:
        with pytest.raises(ValueError):
            O.AbsorbingBC(**kw)


def test_bead_phantom():
    # test/geometry/phantoms.jl:7-43
    g = (101, 101, 96)
    ebg, eb = 1.333 ** 2, 1.4607 ** 2
    ph = O.phantom_bead(g, [eb], 10, permittivity_bg=ebg)
    assert ph.shape == g
    assert ph[0, 0, 0] == pytest.approx(ebg) and ph[-1, -1, -1] == pytest.approx(ebg)
    c = tuple(n // 2 for n in g)  # Julia div(n,2)+1, 1-based
    assert ph[c] == pytest.approx(eb)
    vox = np.count_nonzero(np.abs(ph - eb) < 1e-10)
    assert abs(vox / (4 / 3 * math.pi * 10 ** 3) - 1.0) <= 0.3


def test_phantom_materials_and_edges():
    # test/geometry/phantoms.jl:76-126
    ph = O.phantom_bead((32, 32, 32), [2.25], 8, permittivity_bg=1.0)
    assert np.all(ph.real >= 1.0) and np.all(ph.imag == 0.0)
    ph = O.phantom_bead((32, 32, 32), [2.25 + 0.1j], 8, permittivity_bg=1.0)
    assert ph[16, 16, 16].real == pytest.approx(2.25) and ph[16, 16, 16].imag == pytest.approx(0.1)
    ph = O.phantom_bead((32, 32, 32), [16.0], 5, permittivity_bg=1.0)
    assert ph.real.max() == pytest.approx(16.0)
    small = O.phantom_bead((20, 20, 20), [2.0], 1, permittivity_bg=1.0)
    assert np.count_nonzero(np.abs(small - 2.0) < 1e-10) >= 1
    large = O.phantom_bead((20, 20, 20), [2.0], 15, permittivity_bg=1.0)
    assert np.count_nonzero(np.abs(large - 2.0) < 1e-10) > np.count_nonzero(np.abs(large - 1.0) < 1e-10)


def test_plate_phantom():
    # test/geometry/phantoms.jl:45-74 and 154-173
    eps = (2.9734 + 0.0467j) ** 2
    ph = O.phantom_plate((21, 50, 50), [eps], 4, permittivity_bg=1.0)
    cz = 50 // 2  # Julia div(50,2)+1 -> 0-based 25
    assert ph[9, 24, cz] == pytest.approx(eps)
    assert np.allclose(ph[9, :, cz], ph[9, 24, cz])
    ph2 = O.phantom_plate((20, 20, 20), [2.0], 8, permittivity_bg=1.0)
    assert not np.all(ph2 == 1.0) and ph2.real.max() >= 1.0


def _periodic(res, g):
    return O.SolverConfig((res,) * 3, g, O.PeriodicBC())


def test_plane_wave_shapes_and_finiteness():
    # test/sources/plane_wave.jl:6-33
    cfg = _periodic(50e-9, (64, 64, 32))
    E, H = O.incident_field(O.PlaneWave(532e-9, [1, 0, 0], [0, 0, 1]), cfg)
    assert E.shape == (64, 64, 32, 3) and H.shape == (64, 64, 32, 3)
    assert np.all(np.isfinite(E)) and np.all(np.isfinite(H))


def test_plane_wave_orthogonal_polarisations():
    # test/sources/plane_wave.jl:34-66
    cfg = _periodic(100e-9, (32, 32, 16))
    Ex, _ = O.incident_field(O.PlaneWave(500e-9, [1, 0, 0], [0, 0, 1]), cfg)
    Ey, _ = O.incident_field(O.PlaneWave(500e-9, [0, 1, 0], [0, 0, 1]), cfg)
    O.incident_field(O.PlaneWave(500e-9, [1, 1j, 0], [0, 0, 1]), cfg)
    assert np.sum(np.abs(Ex * np.conj(Ey))) == pytest.approx(0.0, abs=1e-12)


def test_plane_wave_oblique_variation():
    # test/sources/plane_wave.jl:67-96
    cfg = _periodic(10e-9, (20, 50, 50))
    k = np.array([0.0, 0.1, 0.995])
    k = k / np.linalg.norm(k)
    E, _ = O.incident_field(O.PlaneWave(355e-9, [1, 0, 0], k), cfg)
    assert abs(E[10 - 1, 25 - 1, 25 - 1, 0] - E[0, 0, 25 - 1, 0]) > 0.0


def test_plane_wave_impedance():
    # test/sources/plane_wave.jl:97-129 (rtol 0.1 against the free-space impedance)
    cfg = _periodic(50e-9, (32, 32, 32))
    E, H = O.incident_field(O.PlaneWave(633e-9, [1, 0, 0], [0, 0, 1]), cfg)
    c = (16, 16, 16)
    ratio = abs(E[c + (0,)]) / abs(H[c + (1,)])
    assert ratio == pytest.approx(376.730313668, rel=0.1)


def test_plane_wave_superposition():
    # test/sources/plane_wave.jl:130-156
    cfg = _periodic(100e-9, (32, 32, 32))
    s1 = O.PlaneWave(500e-9, [1, 0, 0], [0, 0, 1])
    s2 = O.PlaneWave(500e-9, [0, 1, 0], [0, 0, 1])
    E1, H1 = O.incident_field(s1, cfg)
    E2, H2 = O.incident_field(s2, cfg)
    Et, Ht = O.incident_field([s1, s2], cfg)
    assert Et.shape == (32, 32, 32, 3)
    np.testing.assert_allclose(Et, E1 + E2, rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(Ht, H1 + H2, rtol=1e-14, atol=1e-14)


def test_plane_wave_validation():
    # src/sources/plane_wave.jl:79-90
    with pytest.raises(ValueError):
        O.PlaneWave(500e-9, [1, 0, 0], [0, 0, 2])
    with pytest.raises(ValueError):
        O.PlaneWave(500e-9, [0, 0, 1], [0, 0, 1])
    with pytest.raises(ValueError):
        O.PlaneWave(-1.0, [1, 0, 0], [0, 0, 1])


def test_solver_config_validation_and_roi():
    # test/solvers/convergent_born.jl (construction, validation, domain_size)
    with pytest.raises(ValueError):
        O.SolverConfig((50e-9,) * 3, (32, 32, 32), O.PeriodicBC(), tolerance=2.0)
    with pytest.raises(ValueError):
        O.SolverConfig((-1.0, 1.0, 1.0), (32, 32, 32), O.PeriodicBC())
    bz = O.AbsorbingBC(1e-6, 1e-6, 1.0)
    cfg = O.SolverConfig((50e-9,) * 3, (32, 32, 16), (O.PeriodicBC(), O.PeriodicBC(), bz))
    assert cfg.padded_size == (32, 32, 36)
    assert cfg.roi() == (1, 32, 1, 32, 11, 26)


def test_attenuation_window_quirk():
    # boundary_conditions.jl:638-641: the Tanh window is (tanh(x)/tanh(2.5) - tanh(-2.5))/2
    w = O.attenuation_window(O.TANH, 5)
    assert w[0] == pytest.approx((-1 + math.tanh(2.5)) / 2)
    assert w[-1] == pytest.approx((1 + math.tanh(2.5)) / 2)
    assert w[0] < 0
