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


# The reference's pinned values after two Adam steps on its 4 x 4 grid
# (tests/test_ptyrodactyl/test_multislice/test_multislice_recon.py:185-285):
# potential[0, 0], beam (mode 0)[0, 0], position[0, 0].
PINS = {
    "single_slice_ptychography": (0.02866302842954916, -1.4996974690426799 - 1.4814616332191217j, None),
    "single_slice_poscorrected": (0.02866303668627853, -1.4996974690390232 - 1.4814616332263657j,
                                  0.002001176434824531),
    "single_slice_multi_modal": (0.0286630285066058, -1.4996968965393802 - 1.481462648068354j, 0.0020011719351587594),
    "multi_slice_multi_modal": (0.028663098749764054, -1.4996974690074887 - 1.4814616332889121j, 0.02000915293273863),
}


@pytest.mark.parametrize("n", [4, 16])
@pytest.mark.parametrize("fn", ["single_slice_ptychography", "single_slice_poscorrected", "single_slice_multi_modal",
                                "multi_slice_multi_modal"])
def test_engine_loops_match_the_pinned_oracle_loop(fn, n):
    """The setting of the reference's pinned regressions (PRNGKey(11) draws, two
    positions, 80 kV, unit calibration, two Adam steps at lr 0.001; the oracle's loop
    reproduces those pins on the reference's 4 x 4 grid, tests/test_oracle_recon_pins.py)
    against the same float64 oracle loop: on the reference's own 4 x 4 grid (the
    any-size path), where the reference's pinned scalars are checked as well, and on
    the pass engine's smallest grid, 16 x 16.
    Adam's first steps are lr * sign(g) up to 1e-8, so float32 gradients give the same
    iterates to float32 rounding unless a gradient sits at noise level. That is the
    case for the scan positions here: the object is nearly transparent (|T - 1| ~ 1e-5),
    so the patterns hardly depend on position and the position gradient is a small
    difference of large terms (the oracle's own complex64 and complex128 values of it
    differ by 4-8 %, and the second Adam step with them). The positions are therefore
    held to a quarter of a step: every first step must go the oracle's way (a wrong
    direction is two steps off); well-conditioned position gradients are checked
    against the oracle at 1e-4 in test_gpu_grad.py."""
    from oracle.jax_prng import normal_f64, prng_key, split
    keys = split(prng_key(11), 5)
    pot = (normal_f64(keys[0], (n, n)) * 0.01).astype(np.complex128)
    beam = normal_f64(keys[1], (n, n)) + 1j * normal_f64(keys[2], (n, n))
    modes = np.stack([beam, beam * (0.5 + 0.1j)], axis=-1)
    data = np.ones((2, n, n))
    pos = np.array([[0.0, 0.0], [1.0, 0.0]])
    s4 = pb.create_stem4d(torch.as_tensor(data, dtype=torch.float32, device="cuda"), 1.0, 1.0 / n, pos, 80.0)
    pot_c = pb.create_calibrated_array(pot, 1.0, 1.0, True)
    beam_c = pb.create_calibrated_array(beam, 1.0, 1.0, True)
    lr_pos = 0.01 if fn == "multi_slice_multi_modal" else 0.001
    if fn == "single_slice_ptychography":
        out = MR.single_slice_ptychography(s4, pot_c, beam_c, 1.0, save_every=1, num_iterations=2,
                                           learning_rate=0.001)
        got = (out[0].data_array, out[1].data_array[..., None], None)
        want = R.recon_loop(data, pos, 80.0, 1.0, pot, beam, [1.0], 1.0, 2, 0.001)
    elif fn == "single_slice_poscorrected":
        out = MR.single_slice_poscorrected(s4, pot_c, beam_c, 1.0, save_every=1, num_iterations=2,
                                           learning_rate=0.001)
        got = (out[0].data_array, out[1].data_array[..., None], out[2])
        want = R.recon_loop(data, pos, 80.0, 1.0, pot, beam, [1.0], 1.0, 2, 0.001, lr_pos=0.001)
    elif fn == "single_slice_multi_modal":
        probe = pb.create_probe_modes(modes, [0.7, 0.3], 1.0)
        out = MR.single_slice_multi_modal(s4, pot, probe, 1.0, save_every=1, num_iterations=2, learning_rate=0.001)
        got = (out[0], out[1].modes, out[2])
        want = R.recon_loop(data, pos, 80.0, 1.0, pot, modes, [0.7, 0.3], 1.0, 2, 0.001, lr_pos=0.001)
    else:
        out = MR.multi_slice_multi_modal(s4, pot, beam, 1.0, save_every=1, num_iterations=2, learning_rate=0.001)
        got = (out[0], out[1][..., None], out[2])
        want = R.recon_loop(data, pos, 80.0, 1.0, pot, beam, [1.0], 1.0, 2, 0.001, lr_pos=0.01)
    assert rel_l2(got[0].cpu().numpy(), want["pot"]) < 1e-5
    assert rel_l2(got[1].cpu().numpy(), want["modes"]) < 1e-5
    if got[2] is not None:
        assert np.abs(got[2].cpu().numpy() - want["pos"]).max() < 0.25 * lr_pos
    if n == 4:
        pin_pot, pin_beam, pin_pos = PINS[fn]
        assert abs(complex(got[0][0, 0].item()) - pin_pot) <= 1e-5 * abs(pin_pot)
        assert abs(complex(got[1][0, 0, 0].item()) - pin_beam) <= 1e-5 * abs(pin_beam)
        if pin_pos is not None:
            assert abs(float(got[2][0, 0]) - pin_pos) < 0.25 * lr_pos
