"""The reference's public per-step functions (transmission_func, propagation_func,
shift_beam_fourier, fourier_coords, fourier_calib) against the oracle's
restatements, on square, rectangular and odd grids. CPU only."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R


def test_transmission_func():
    v = np.random.default_rng(0).uniform(0.0, 40.0, (7, 12))
    got = pb.transmission_func(v, 200.0)
    assert got.dtype == torch.complex128 and tuple(got.shape) == (7, 12)
    assert np.allclose(got.numpy(), R.transmission_func(v, 200.0), rtol=0, atol=1e-14)


@pytest.mark.parametrize("h,w", [(16, 16), (24, 40), (7, 5)])
def test_propagation_func(h, w):
    got = pb.propagation_func(h, w, 1.7, 300.0, 0.23)
    assert got.dtype == torch.complex128 and tuple(got.shape) == (h, w)
    assert np.allclose(got.numpy(), R.propagation_func(h, w, 1.7, 300.0, 0.23), rtol=0, atol=1e-13)


@pytest.mark.parametrize("shape", [(16, 16, 2), (24, 40, 1), (9, 6)])
def test_shift_beam_fourier(shape):
    rng = np.random.default_rng(len(shape))
    beam = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    pos = rng.uniform(-3, 3, (4, 2))
    got = pb.shift_beam_fourier(beam, pos, 0.3)
    want = R.shift_beam_fourier(beam, pos, 0.3)
    assert got.dtype == torch.complex128 and tuple(got.shape) == want.shape
    assert np.allclose(got.numpy(), want, rtol=0, atol=1e-12)
    # an integer-pixel shift (in units of calib) is a circular roll
    roll = pb.shift_beam_fourier(beam, [[2 * 0.3, -1 * 0.3]], 0.3)[0].numpy()
    b3 = beam if beam.ndim == 3 else beam[..., None]
    assert np.allclose(roll, np.roll(b3, (2, -1), axis=(0, 1)), atol=1e-12)


@pytest.mark.parametrize("size,calib", [((16, 16), 0.25), ((24, 40), 0.1), ((7, 5), 0.5)])
def test_fourier_coords_and_calib(size, calib):
    fc = pb.fourier_coords(calib, size)
    want = R.probe_fourier_radius(size, calib * 100.0)
    assert np.allclose(fc.data_array.numpy(), want, rtol=0, atol=1e-13)
    assert not fc.real_space
    assert np.isclose(fc.calib_y, 1.0 / (size[0] * calib)) and np.isclose(fc.calib_x, 1.0 / (size[1] * calib))
    cal = pb.fourier_calib(calib, size).numpy()
    assert np.allclose(cal, [1.0 / (size[0] * calib), 1.0 / (size[1] * calib)])


def test_building_blocks_are_differentiable():
    v = torch.rand(6, 8, dtype=torch.float64, requires_grad=True)
    t = pb.transmission_func(v, 200.0)
    t.real.sum().backward()
    sigma = pb.interaction_sigma(200.0)
    assert torch.allclose(v.grad, -sigma * torch.sin(sigma * v.detach()))
    pos = torch.tensor([[0.4, -0.7]], dtype=torch.float64, requires_grad=True)
    beam = torch.randn(8, 8, dtype=torch.complex128)
    pb.shift_beam_fourier(beam, pos, 0.3).abs().pow(2).sum().backward()
    assert pos.grad is not None and bool(torch.isfinite(pos.grad).all())


def test_physics_helpers_match_the_reference_values():
    """types/constants.py:119-288: sigma 0.92440e-3 / 0.65262e-3 rad/(V A) and sigma_H
    0.31383 / 0.41656 1/(V A^2) at 100 / 300 kV; sigma_H = 2 k0 sigma; sigma is the
    transmission's interaction constant."""
    for kv, sig, sh in [(100.0, 0.92440e-3, 0.31383), (300.0, 0.65262e-3, 0.41656)]:
        s = pb.phase_interaction_parameter(kv)
        h = pb.helmholtz_coupling(kv)
        assert abs(s - sig) < 5e-9 and abs(h - sh) < 5e-6
        k0 = 2.0 * np.pi / pb.relativistic_wavelength_ang(kv)
        assert np.isclose(h, 2.0 * k0 * s, rtol=1e-14, atol=0.0)
        assert np.isclose(s, pb.interaction_sigma(kv), rtol=1e-14, atol=0.0)
    assert np.isclose(pb.relativistic_mass(0.0), pb.M_E, rtol=0, atol=0)
    assert np.isclose(pb.relativistic_mass(pb.M0C2_EV / 1000.0), 2.0 * pb.M_E, rtol=1e-8)
