"""Sub-pixel atom placement of crystal_potential_slices on the GPU against the
oracle's per-atom Fourier-shift restatement."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _gaussian(n, width):
    c = np.arange(n) - n / 2.0
    yy, xx = np.meshgrid(c, c, indexing="ij")
    return np.exp(-(xx ** 2 + yy ** 2) / (2 * width ** 2))


def _perovskite(a=3.905):
    frac = np.array([[0, 0, 0], [0.5, 0.5, 0.5], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    return frac * a, np.array([38, 22, 8, 8, 8]), np.eye(3) * a


@pytest.mark.parametrize("n,reps,thick", [(64, (3, 3, 2), 1.95), (128, (6, 5, 1), 3.905)])
def test_crystal_potential_slices_match_oracle(n, reps, thick):
    pos, nums, lat = _perovskite()
    rng = np.random.default_rng(n)
    pos = pos + rng.normal(0, 0.05, pos.shape)
    lookup = {38: 9.0 * _gaussian(n, 2.5), 22: 6.0 * _gaussian(n, 2.0), 8: 2.5 * _gaussian(n, 1.5)}
    crystal = pb.create_crystal_data(pos, nums, lat)
    px = 0.25
    s_out = int(np.floor((pos[:, 2].max() + (reps[2] - 1) * 3.905 - pos[:, 2].min()) / thick)) + 1
    got = pb.crystal_potential_slices(crystal, px, thick, reps, padding=2.0, grid_shape=(n, n, s_out),
                                      atom_potentials=lookup)
    want = R.crystal_potential_slices(pos, nums, lat, lookup, px, thick, reps, padding=2.0, grid_shape=(n, n, s_out))
    data = got.slices.cpu().numpy()
    assert data.shape == want.shape
    assert rel_l2(data, want) < 1e-5, rel_l2(data, want)
    assert got.calib == px and got.slice_thickness == thick


def test_crystal_potential_slices_errors():
    pos, nums, lat = _perovskite()
    with pytest.raises(ValueError, match="CrystalData.lattice must not be None"):
        pb.crystal_potential_slices(pb.create_crystal_data(pos, nums), 0.25, atom_potentials={})
    with pytest.raises(ValueError, match="parameterization must be 'lobato' or 'kirkland'"):
        pb.crystal_potential_slices(pb.create_crystal_data(pos, nums, lat), 0.25, grid_shape=(64, 64, 2),
                                    parameterization="doyle")
    with pytest.raises(ValueError, match="pass grid_shape"):
        pb.crystal_potential_slices(pb.create_crystal_data(pos, nums, lat), 0.25, atom_potentials={38: 1})
    with pytest.raises(ValueError, match="positions must have shape"):
        pb.create_crystal_data(np.zeros((3, 2)), [1, 2, 3])


@pytest.mark.parametrize("z,expected_sum,expected_max", [(6, 3304.630500664369, 599.0660669230273),
                                                         (14, 7467.50633667953, 1309.8209272295387),
                                                         (79, 16835.066119859865, 6296.83419348897)])
def test_single_atom_potential_kirkland_matches_captured_reference(z, expected_sum, expected_max):
    """The reference's captured Kirkland values for C, Si and Au (0.2 A pixels, 16 x 16,
    supersampling 2; tests/test_ptyrodactyl/test_multislice/test_atom_potentials.py:31-63)
    from the device kernel, in float64."""
    got = pb.single_atom_potential(z, 0.2, (16, 16), supersampling=2, parameterization="kirkland")
    assert got.dtype == torch.float64 and got.is_cuda
    assert abs(float(got.sum()) - expected_sum) <= 1e-13 * expected_sum
    assert abs(float(got.max()) - expected_max) <= 1e-13 * expected_max


@pytest.mark.parametrize("parameterization", ["lobato", "kirkland"])
@pytest.mark.parametrize("z,shape,center,s", [(1, (16, 24), None, 4), (38, (64, 64), (0.3, -0.7), 3),
                                              (79, (32, 32), (1.1, 0.25), 1), (103, (20, 12), None, 2)])
def test_single_atom_potential_matches_oracle(parameterization, z, shape, center, s):
    got = pb.single_atom_potential(z, 0.15, shape, center, s, parameterization=parameterization).cpu().numpy()
    want = R.single_atom_potential(z, 0.15, shape, center, s, parameterization=parameterization)
    assert got.shape == want.shape
    assert np.allclose(got, want, rtol=1e-12, atol=0.0)


def test_crystal_potential_slices_builds_its_own_lookups():
    """Without atom_potentials the per-element lookups are the device-evaluated Lobato
    potentials at the padded grid's centre, as in the reference (atom_potentials.py
    :1290-1312); the slices match the oracle built from the oracle's own lookups."""
    pos, nums, lat = _perovskite()
    n, px, thick, reps = 64, 0.25, 1.95, (3, 3, 2)
    rng = np.random.default_rng(4)
    pos = pos + rng.normal(0, 0.05, pos.shape)
    crystal = pb.create_crystal_data(pos, nums, lat)
    s_out = int(np.floor((pos[:, 2].max() + (reps[2] - 1) * 3.905 - pos[:, 2].min()) / thick)) + 1
    got = pb.crystal_potential_slices(crystal, px, thick, reps, padding=2.0, supersampling=2,
                                      grid_shape=(n, n, s_out))
    lookup = {z: R.single_atom_potential(z, px, (n, n), (0.0, 0.0), 2) for z in (8, 22, 38)}
    want = R.crystal_potential_slices(pos, nums, lat, lookup, px, thick, reps, padding=2.0, grid_shape=(n, n, s_out))
    assert rel_l2(got.slices.cpu().numpy(), want) < 1e-5
