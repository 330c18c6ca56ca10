"""The oracle's reconstruction loops against the reference's own pinned values.

The reference pins its four gradient-based loops as float64 scalars after two Adam
steps on a 4 x 4 grid (tests/test_ptyrodactyl/test_multislice/test_multislice_recon.py
:185-285), with inputs drawn from ``jax.random.PRNGKey(11)`` (:35-62). Reproducing
them checks the oracle's forward model, its hand-derived gradients (potential, beam
and scan positions) and the optimizer restatement against values the reference
computed with ``jax.value_and_grad`` through ``stem_4d``. JAX draws the inputs with
``split`` and ``normal`` (``oracle/jax_prng.py``); XLA's ``erf_inv`` is not restated
bit for bit, so the comparison allows a few units in the last place (relative 1e-12;
the positions, which move by Adam steps of 1e-3 from zero, 1e-10).
"""

import numpy as np
import pytest

from oracle import multislice_ref as R
from oracle.jax_prng import erfinv, normal_f64, prng_key, split

RTOL = 1e-12
RTOL_POS = 1e-10


@pytest.fixture(scope="module")
def tiny():
    """_tiny_recon_inputs (test_multislice_recon.py:35-62)."""
    keys = split(prng_key(11), 5)
    pot = (normal_f64(keys[0], (4, 4)) * 0.01).astype(np.complex128)
    beam = normal_f64(keys[1], (4, 4)) + 1j * normal_f64(keys[2], (4, 4))
    modes = np.stack([beam, beam * (0.5 + 0.1j)], axis=-1)
    data = np.ones((2, 4, 4))
    pos = np.array([[0.0, 0.0], [1.0, 0.0]])
    return data, pos, pot, beam, modes


def _close(got, want, rtol):
    assert abs(got - want) <= rtol * abs(want), (got, want)


def test_erfinv_matches_scipy():
    sp = pytest.importorskip("scipy.special")
    ys = np.concatenate([np.linspace(-0.999999, 0.999999, 4001), [1e-300, -1e-17, 0.9999999999999999]])
    for y in ys:
        want = float(sp.erfinv(y))
        assert abs(erfinv(y) - want) <= 2e-15 * max(abs(want), 1e-300), y


def test_split_keys_are_distinct_threefry_blocks():
    keys = split(prng_key(11), 5)
    assert len(set(keys)) == 5
    assert all(0 <= k < 2 ** 32 for key in keys for k in key)


def test_single_slice_ptychography_pins(tiny):
    """test_single_slice_ptychography_runs_and_regresses (:185-206)."""
    data, pos, pot, beam, _ = tiny
    r = R.recon_loop(data, pos, 80.0, 1.0, pot, beam, [1.0], 1.0, 2, 0.001)
    assert r["snap_pot"].shape == (4, 4, 2) and r["snap_modes"].shape == (4, 4, 1, 2)
    _close(r["pot"][0, 0], 0.02866302842954916 + 0j, RTOL)
    _close(r["modes"][0, 0, 0], -1.4996974690426799 - 1.4814616332191217j, RTOL)
    _close(r["snap_pot"][0, 0, 0], 0.027663112105862656 + 0j, RTOL)


def test_single_slice_poscorrected_pins(tiny):
    """test_single_slice_poscorrected_regresses (:209-230): one learning rate for the
    parameters and the positions."""
    data, pos, pot, beam, _ = tiny
    r = R.recon_loop(data, pos, 80.0, 1.0, pot, beam, [1.0], 1.0, 2, 0.001, lr_pos=0.001)
    _close(r["pot"][0, 0], 0.02866303668627853 + 0j, RTOL)
    _close(r["modes"][0, 0, 0], -1.4996974690390232 - 1.4814616332263657j, RTOL)
    _close(r["pos"][0, 0], 0.002001176434824531, RTOL_POS)


def test_single_slice_multi_modal_pins(tiny):
    """test_single_slice_multi_modal_regresses (:233-258): two modes, weights 0.7 / 0.3."""
    data, pos, pot, _, modes = tiny
    r = R.recon_loop(data, pos, 80.0, 1.0, pot, modes, [0.7, 0.3], 1.0, 2, 0.001, lr_pos=0.001)
    assert r["snap_modes"].shape == (4, 4, 2, 2)
    _close(r["pot"][0, 0], 0.0286630285066058 + 0j, RTOL)
    _close(r["modes"][0, 0, 0], -1.4996968965393802 - 1.481462648068354j, RTOL)
    _close(r["pos"][0, 0], 0.0020011719351587594, RTOL_POS)


def test_multi_slice_multi_modal_pins(tiny):
    """test_multi_slice_multi_modal_regresses (:261-285): positions step with the
    default position learning rate 0.01."""
    data, pos, pot, beam, _ = tiny
    r = R.recon_loop(data, pos, 80.0, 1.0, pot, beam, [1.0], 1.0, 2, 0.001, lr_pos=0.01)
    _close(r["pot"][0, 0], 0.028663098749764054 + 0j, RTOL)
    _close(r["modes"][0, 0, 0], -1.4996974690074887 - 1.4814616332889121j, RTOL)
    _close(r["pos"][0, 0], 0.02000915293273863, RTOL_POS)
