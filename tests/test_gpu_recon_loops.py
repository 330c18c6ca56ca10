"""The reference's reconstruction loops on the engine: a few Adam iterations of
single_slice_poscorrected against the oracle's float64 loop, and the other loops'
shapes, snapshots and progress."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from ptyrodactyl_b200 import multislice_recon as MR
from oracle import multislice_ref as R
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _problem(n=32, p=9, seed=2):
    rng = np.random.default_rng(seed)
    calib = 0.25
    truth = rng.uniform(0, 20, (n, n))
    probe = R.make_probe(200.0, 25.0, (n, n), calib * 100, defocus_ang=-30.0)
    pos = rng.uniform(-1.5, 1.5, (p, 2))
    data = R.stem_4d(truth[..., None], 2.0, calib, probe[..., None], [1.0], calib, 200.0, pos, calib)["data"]
    s4 = pb.create_stem4d(torch.as_tensor(data, dtype=torch.float32, device="cuda"), calib, 1.0 / (n * calib), pos,
                          200.0)
    pot0 = truth + rng.normal(0, 1.0, truth.shape)
    beam0 = probe * np.exp(0.1j)
    return s4, data, pos, pot0, beam0, calib


def test_poscorrected_matches_oracle_loop():
    s4, data, pos, pot0, beam0, calib = _problem()
    its, lr, lr_pos = 3, 0.05, 0.01
    pot, beam, got_pos, sp, sb, spos = MR.single_slice_poscorrected(
        s4, pb.create_calibrated_array(pot0, calib, calib, True), pb.create_calibrated_array(beam0, calib, calib, True),
        2.0, save_every=1, num_iterations=its, learning_rate=(lr, lr_pos))
    want_pot, want_beam, want_pos, losses = R.single_slice_poscorrected(data, pos, 200.0, calib, pot0, beam0, 2.0,
                                                                        its, lr, lr_pos)
    # Adam's first steps are close to lr * sign(g): the few pixels whose gradient is at
    # float32 noise level may step the other way, so compare the iterates themselves
    assert rel_l2(pot.data_array.cpu().numpy(), want_pot) < 2e-3
    assert rel_l2(beam.data_array.cpu().numpy(), want_beam) < 1e-2  # small-amplitude pixels move by lr
    assert rel_l2(got_pos.cpu().numpy(), want_pos) < 2e-3
    got_loss = float(np.mean((R.stem_4d(np.real(pot.data_array.cpu().numpy())[..., None], 2.0, calib,
                                        beam.data_array.cpu().numpy()[..., None], [1.0], calib, 200.0,
                                        got_pos.cpu().numpy(), calib)["data"] - data) ** 2))
    want_loss = float(np.mean((R.stem_4d(np.real(want_pot)[..., None], 2.0, calib, want_beam[..., None], [1.0],
                                         calib, 200.0, want_pos, calib)["data"] - data) ** 2))
    assert abs(got_loss - want_loss) <= 0.02 * want_loss
    assert sp.shape == pot0.shape + (its,) and spos.shape == (len(pos), 2, its)
    assert torch.equal(sp[..., -1], pot.data_array)


@pytest.mark.parametrize("fn", ["single_slice_ptychography", "single_slice_multi_modal", "multi_slice_multi_modal"])
def test_reconstruction_loops_reduce_the_loss(fn):
    s4, data, pos, pot0, beam0, calib = _problem(seed=5)
    rng = np.random.default_rng(8)
    truth_like = pot0  # a perturbed potential with the exact beam: the loops must lower the loss
    beam0 = R.make_probe(200.0, 25.0, pot0.shape, calib * 100, defocus_ang=-30.0)
    pot0 = truth_like + rng.normal(0, 20.0, pot0.shape)

    def loss_of(pot, beam_modes, positions):
        model = R.stem_4d(np.real(pot)[..., None], 2.0, calib, beam_modes, [1.0] * beam_modes.shape[-1], calib,
                          200.0, positions, calib)["data"]
        return float(np.mean((model - data) ** 2))

    start = loss_of(pot0, beam0[..., None], pos)
    if fn == "single_slice_ptychography":
        pot, beam, sp, sb = MR.single_slice_ptychography(
            s4, pb.create_calibrated_array(pot0, calib, calib, True),
            pb.create_calibrated_array(beam0, calib, calib, True), 2.0, save_every=5, num_iterations=12,
            learning_rate=1e-4)
        end = loss_of(pot.data_array.cpu().numpy(), beam.data_array.cpu().numpy()[..., None], pos)
        assert sp.shape[-1] == 2 and torch.equal(sp[..., 0] != 0, torch.ones_like(sp[..., 0], dtype=torch.bool))
    elif fn == "single_slice_multi_modal":
        beam = pb.create_probe_modes(beam0[..., None], [1.0], calib)
        pot, probe, p2, sp, sm = MR.single_slice_multi_modal(s4, pot0, beam, 2.0, save_every=4, num_iterations=12,
                                                             learning_rate=(1e-4, 1e-4))
        end = loss_of(pot.cpu().numpy(), probe.modes.cpu().numpy(), p2.cpu().numpy())
        assert sm.shape == beam0.shape + (1, 3)
    else:
        pot, b, p2, sp, sb = MR.multi_slice_multi_modal(s4, pot0, beam0, 2.0, save_every=4, num_iterations=12,
                                                        learning_rate=1e-4, pos_learning_rate=1e-4)
        end = loss_of(pot.cpu().numpy(), b.cpu().numpy()[..., None], p2.cpu().numpy())
    assert end < start


def test_unknown_optimizer_and_loss():
    s4, data, pos, pot0, beam0, calib = _problem()
    with pytest.raises(ValueError, match="Unknown optimizer"):
        MR.multi_slice_multi_modal(s4, pot0, beam0, 2.0, num_iterations=1, optimizer_name="sgd")
    with pytest.raises(ValueError):
        MR.multi_slice_multi_modal(s4, pot0, beam0, 2.0, num_iterations=1, loss_type="huber")
