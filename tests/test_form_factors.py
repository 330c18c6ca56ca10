"""Form factors and projected potentials of single atoms (form_factors.py): the
reference's physics checks (tests/test_ptyrodactyl/test_multislice/test_form_factors.py),
the oracle's restatement, and SciPy's Bessel functions. CPU only."""

import numpy as np
import pytest
import torch

from oracle import multislice_ref as R
from ptyrodactyl_b200 import form_factors as FF


def test_hydrogen_zero_angle_form_factor_is_bohr_radius():
    """The neutral-H Bethe anchor f_H(0) = a_0."""
    assert np.isclose(float(FF.atomic_form_factor(1, 0.0)), FF.A_BOHR, rtol=1e-9, atol=0.0)


@pytest.mark.parametrize("z,g_max,volts", [(6, 2.0, 417.0), (6, 3.0, 712.0), (6, 4.0, 1028.0),
                                           (14, 2.0, 823.0), (14, 3.0, 1513.0), (14, 4.0, 2238.0),
                                           (79, 2.0, 3327.0), (79, 3.0, 6534.0), (79, 4.0, 10125.0)])
def test_bandlimited_peaks_match_published_table(z, g_max, volts):
    assert abs(float(FF.lobato_bandlimited_peak(z, g_max)) - volts) <= 0.51


@pytest.mark.parametrize("z", [6, 14, 79])
def test_parameterizations_agree(z):
    """Form factors within 0.6 % over g = 0..4 / A; projected potentials within 3 % over
    r = 0.05..1.5 A."""
    q = 2.0 * np.pi * np.linspace(0.0, 4.0, 201)
    lob = FF.atomic_form_factor(z, q, parameterization="lobato").numpy()
    kir = FF.atomic_form_factor(z, q, parameterization="kirkland").numpy()
    assert np.allclose(kir, lob, rtol=6e-3, atol=0.0)
    r = np.geomspace(0.05, 1.5, 201)
    lob = FF.projected_atom_potential(z, r, parameterization="lobato").numpy()
    kir = FF.projected_atom_potential(z, r, parameterization="kirkland").numpy()
    assert np.allclose(kir, lob, rtol=3e-2, atol=0.0)


@pytest.mark.parametrize("parameterization", ["lobato", "kirkland"])
def test_projected_potential_matches_oracle(parameterization):
    r = np.geomspace(1e-3, 4.0, 97)
    for z in (1, 8, 29, 79):
        got = FF.projected_atom_potential(z, r, parameterization=parameterization).numpy()
        want = R.projected_potential(R.element_coefficients(z, parameterization), r, parameterization)
        assert np.allclose(got, want, rtol=1e-12, atol=0.0)


def test_bessel_kv_against_scipy():
    from scipy.special import kv
    x = np.geomspace(0.01, 30.0, 200)
    for v, tol in [(0.0, 2e-7), (1.0, 2e-7), (0.5, 1e-14), (2.0, 1e-14), (1.3, 1e-14)]:
        got = FF.bessel_kv(v, x).numpy()
        assert np.allclose(got, kv(v, x), rtol=tol, atol=0.0), v


def test_validation():
    with pytest.raises(ValueError, match="parameterization"):
        FF.atomic_form_factor(6, 1.0, parameterization="doyle")
    with pytest.raises(ValueError):
        FF.projected_atom_potential(0, 1.0)
    with pytest.raises(ValueError):
        FF.atomic_form_factor(True, 1.0)
    with pytest.raises(ValueError, match="nonnegative"):
        FF.projected_atom_potential(6, [-0.1, 1.0])
    with pytest.raises(ValueError, match="positive and finite"):
        FF.lobato_bandlimited_peak(6, 0.0)
    with pytest.raises(ValueError, match="positive"):
        FF.create_lobato_parameters(np.ones(5), -np.ones(5))
    p = FF.create_kirkland_parameters(np.ones(3), np.ones(3), np.ones(3), np.ones(3))
    assert isinstance(FF.kirkland_form_factor(p, torch.zeros(4)), torch.Tensor)
