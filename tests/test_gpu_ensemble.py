"""Ensemble axes (probe modes, position jitter, partial coherence) and complex
amplitudes on the GPU, against the oracle's restatement of cbed_image's ensemble
branch."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _setup(n=64, s=4, m=2, seed=3):
    rng = np.random.default_rng(seed)
    pot = rng.uniform(0.0, 40.0, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 25.0, defocus_ang=-30.0)
    modes = probe[..., None] if m == 1 else np.stack([probe, np.roll(probe, 2, axis=1) * (0.8 - 0.2j)], -1)
    w = np.array([1.0]) if m == 1 else np.array([0.65, 0.35])
    return pot, modes, w


def _axes_oracle(d):
    return (d.samples.numpy(), d.weights.numpy(), d.reduction.value, d.axis_id)


def test_cbed_amplitude_matches_oracle():
    pot, modes, w = _setup()
    pots = pb.create_potential_slices(pot, 1.7, 0.25)
    beam = pb.create_probe_modes(modes, w, 0.25)
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(64, 64))
    got = pb.cbed_amplitude(pots, beam, mic)
    assert got.shape == (64, 64, 2) and got.dtype == torch.complex64
    want = R.cbed_amplitude(pot, 1.7, 200.0, 0.25, modes)
    assert rel_l2(got.cpu().numpy(), want) < TOL
    # the incoherent sum of the amplitudes is cbed_image
    img = pb.cbed_image(pots, beam, mic).data_array
    inten = (got.abs() ** 2 * torch.as_tensor(w, dtype=torch.float32, device=got.device)).sum(-1)
    assert torch.allclose(img, inten, rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("jitter,energy,tilt,m", [(0.12, 0.0, 0.0, 1), (0.0, 0.8, 0.3, 1), (0.1, 0.6, 0.2, 2),
                                                  (0.0, 0.0, 0.0, 2)])
def test_cbed_image_ensemble_matches_oracle(jitter, energy, tilt, m):
    pot, modes, w = _setup(m=m)
    ens = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(jitter, 2),
                                  coherence=pb.coherence_to_distribution(energy, tilt, 2))
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(64, 64))
    beam = pb.create_probe_modes(modes, w, 0.25)
    got = pb.cbed_image(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic).data_array.cpu().numpy()
    axes = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens, beam)]
    want = R.ensemble_cbed(pot, 1.7, 0.25, modes, 0.25, 200.0, axes)
    assert rel_l2(got, want) < TOL, rel_l2(got, want)


def test_stem_4d_ensemble_matches_oracle():
    pot, modes, w = _setup(n=64, s=3, m=2, seed=8)
    pos = np.random.default_rng(1).uniform(-2, 2, (5, 2))
    ens = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(0.08, 2),
                                  coherence=pb.coherence_to_distribution(0.5, 0.15, 2))
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(64, 64))
    beam = pb.create_probe_modes(modes, w, 0.25)
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    s4 = pb.stem_4d(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic, det)
    axes = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens, beam)]
    want = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes)
    assert rel_l2(s4.data.cpu().numpy(), want) < TOL


def test_coherent_mode_axis_and_unsupported_coherent_tilts():
    pot, modes, w = _setup(m=2)
    coh = pb.create_distribution(np.arange(2.0)[:, None], w, pb.ReductionMode.COHERENT, "probe_modes")
    ens = pb.create_ensemble_axes(probe_modes=coh)
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(64, 64))
    beam = pb.create_probe_modes(modes, w, 0.25)
    got = pb.cbed_image(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic).data_array.cpu().numpy()
    want = R.ensemble_cbed(pot, 1.7, 0.25, modes, 0.25, 200.0, [_axes_oracle(coh)])
    assert rel_l2(got, want) < TOL
    c = pb.coherence_to_distribution(0.5, 0.2, 2)
    coherent_tilts = pb.create_distribution(c.samples, c.weights, pb.ReductionMode.COHERENT, "coherence")
    ens2 = pb.create_ensemble_axes(probe_modes=coh, coherence=coherent_tilts)
    mic2 = pb.create_microscope_config(200.0, 25.0, ensemble=ens2, probe_shape=(64, 64))
    with pytest.raises(NotImplementedError, match="coherent sums over energy or tilt"):
        pb.cbed_image(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic2)
