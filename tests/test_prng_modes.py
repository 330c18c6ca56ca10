"""decompose_beam_to_modes and the JAX-key draws behind it, against the reference's
own pinned values (tests/test_ptyrodactyl/test_multislice/test_simulations.py:125-216)
and the oracle's independent restatement of JAX's generator. CPU only."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import jax_prng as J
from ptyrodactyl_b200 import prng


def _beam():
    return pb.create_calibrated_array((np.arange(16, dtype=np.float64).reshape(4, 4) + 1j).astype(np.complex128),
                                      0.5, 0.5, True)


def test_draws_match_the_oracle_generator():
    for seed in (0, 11, 42, 2 ** 40 + 3):
        k = prng.prng_key(seed)
        assert k == J.prng_key(seed)
        assert prng.split(k, 3) == J.split(k, 3)
        assert np.array_equal(prng.uniform(k, (7, 5)), J.uniform_f64(k, (7, 5)))
        assert np.max(np.abs(prng.normal(k, (64,)) - J.normal_f64(k, (64,)))) < 1e-15


def test_fixed_key_reproduces_the_pinned_mode():
    """PRNGKey(0), three modes: the reference pins modes[0, 0, 0] and the weights."""
    first = pb.decompose_beam_to_modes(_beam(), 3, prng.prng_key(0), first_mode_weight=0.6)
    second = pb.decompose_beam_to_modes(_beam(), 3, 0, first_mode_weight=0.6)
    assert torch.equal(first.modes, second.modes) and torch.equal(first.weights, second.weights)
    assert first.modes.dtype == torch.complex128 and tuple(first.modes.shape) == (4, 4, 3)
    # the reference's value, to the few units in the last place its erfinv and QR
    # rounding allow
    assert abs(complex(first.modes[0, 0, 0]) - (-0.34562459928563927 + 0.25753846176370626j)) < 1e-14
    assert np.allclose(first.weights.numpy(), [0.6, 0.2, 0.2])
    assert float(first.calib) == 0.5
    w = first.weights.to(torch.float64)
    weighted = torch.einsum("m,hwm->hw", w, first.modes.abs() ** 2)
    prescaled = ((first.modes * w.sqrt().reshape(1, 1, -1)).abs() ** 2).sum(-1)
    assert torch.allclose(weighted, prescaled, rtol=1e-15, atol=1e-15)
    # orthonormal columns before the amplitude scaling
    q = first.modes.reshape(16, 3) / torch.from_numpy(np.abs(_beam().data_array.numpy()).reshape(16, 1))
    assert torch.allclose(q.conj().T @ q, torch.eye(3, dtype=torch.complex128), atol=1e-12)


def test_single_mode_and_missing_key():
    one = pb.create_calibrated_array(np.ones((4, 4), np.complex128), 0.5, 0.5, True)
    r = pb.decompose_beam_to_modes(one, 1, prng.prng_key(3))
    assert tuple(r.modes.shape) == (4, 4, 1) and np.array_equal(r.weights.numpy(), [1.0])
    with pytest.raises(TypeError):
        pb.decompose_beam_to_modes(_beam(), 3)
