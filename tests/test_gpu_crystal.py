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
    with pytest.raises(NotImplementedError, match="pass atom_potentials"):
        pb.crystal_potential_slices(pb.create_crystal_data(pos, nums, lat), 0.25, grid_shape=(64, 64, 2))
    with pytest.raises(ValueError, match="pass grid_shape"):
        pb.crystal_potential_slices(pb.create_crystal_data(pos, nums, lat), 0.25, atom_potentials={38: 1})
    with pytest.raises(ValueError, match="positions must have shape"):
        pb.create_crystal_data(np.zeros((3, 2)), [1, 2, 3])
