"""Ensemble axes (probe modes, position jitter, partial coherence) and complex
amplitudes on the GPU, against the oracle's restatement of cbed_image's ensemble
branch."""

import dataclasses

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


def test_coherent_mode_axis_and_coherent_energy_tilt_sums():
    pot, modes, w = _setup(m=2)
    coh = pb.create_distribution(np.arange(2.0)[:, None], w, pb.ReductionMode.COHERENT, "probe_modes")
    ens = pb.create_ensemble_axes(probe_modes=coh)
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(64, 64))
    beam = pb.create_probe_modes(modes, w, 0.25)
    got = pb.cbed_image(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic).data_array.cpu().numpy()
    want = R.ensemble_cbed(pot, 1.7, 0.25, modes, 0.25, 200.0, [_axes_oracle(coh)])
    assert rel_l2(got, want) < TOL
    # a COHERENT coherence axis (energy and tilt samples summed as amplitudes), with
    # the coherent mode axis, in cbed_image; and with an incoherent jitter axis in stem_4d
    c = pb.coherence_to_distribution(0.5, 0.2, 2)
    coherent_tilts = pb.create_distribution(c.samples, c.weights, pb.ReductionMode.COHERENT, "coherence")
    ens2 = pb.create_ensemble_axes(probe_modes=coh, coherence=coherent_tilts)
    mic2 = pb.create_microscope_config(200.0, 25.0, ensemble=ens2, probe_shape=(64, 64))
    got2 = pb.cbed_image(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic2).data_array.cpu().numpy()
    axes2 = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens2, beam)]
    want2 = R.ensemble_cbed(pot, 1.7, 0.25, modes, 0.25, 200.0, axes2)
    assert rel_l2(got2, want2) < TOL
    ens3 = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(0.06, 2),
                                   coherence=coherent_tilts)
    mic3 = pb.create_microscope_config(200.0, 25.0, ensemble=ens3, probe_shape=(64, 64))
    beam1 = pb.create_probe_modes(modes[..., :1], np.array([1.0]), 0.25)
    pos = np.random.default_rng(3).uniform(-2, 2, (4, 2))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    s4 = pb.stem_4d(pb.create_potential_slices(pot, 1.7, 0.25), beam1, mic3, det)
    axes3 = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens3, beam1)]
    want3 = R.stem_4d_ensemble(pot, 1.7, 0.25, modes[..., :1], 0.25, 200.0, pos, 0.3, axes3)
    assert rel_l2(s4.data.cpu().numpy(), want3) < TOL
    # any-size grids have no amplitude forward at scan positions: refused by name
    mic4 = pb.create_microscope_config(200.0, 25.0, ensemble=ens2, probe_shape=(40, 56))
    rect = np.random.default_rng(1).uniform(0.0, 20.0, (40, 56, 2))
    probe = R.make_probe(200.0, 25.0, (40, 56), 25.0)
    beam2 = pb.create_probe_modes(np.stack([probe, probe * 0.5j], -1), w, 0.25)
    with pytest.raises(NotImplementedError, match="coherent sums over energy or tilt"):
        pb.cbed_image(pb.create_potential_slices(rect, 1.7, 0.25), beam2, mic4)


@pytest.mark.parametrize("jitter,energy", [(0.08, 0.0), (0.0, 0.6), (0.1, 0.5)])
def test_stem_4d_ensemble_gradients_match_oracle(jitter, energy):
    """Reverse mode through incoherent jitter and energy-spread axes and a two-mode
    beam: the patterns against the oracle's ensemble branch, and dL/dV, dL/dbeam,
    dL/d(weights) and dL/d(positions) against the oracle's adjoint summed over the
    (energy, jitter) samples, each at the scan positions moved by the jitter (the
    jitter's Fourier shift at the beam calibration composed with the scan shift)."""
    pot, modes, w = _setup(n=64, s=3, m=2, seed=12)
    rng = np.random.default_rng(4)
    pos = rng.uniform(-2, 2, (4, 2))
    g = rng.normal(size=(4, 64, 64))
    ens = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(jitter, 2),
                                  coherence=pb.coherence_to_distribution(energy, 0.0, 2))
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(64, 64))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    dev = torch.device("cuda")
    V = torch.tensor(pot, dtype=torch.float32, device=dev, requires_grad=True)
    md = torch.tensor(modes.astype(np.complex64), device=dev, requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float32, device=dev, requires_grad=True)
    ps = torch.tensor(pos, dtype=torch.float64, device=dev, requires_grad=True)
    det_t = dataclasses.replace(det, scan_positions_px=ps)
    s4 = pb.stem_4d(pb.PotentialSlices(V, 1.7, 0.25), pb.ProbeModes(md, wt, 0.25), mic, det_t)
    (s4.data * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()
    beam = pb.create_probe_modes(modes, w, 0.25)
    axes = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens, beam)]
    want = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes)
    assert rel_l2(s4.data.detach().cpu().numpy(), want) < TOL
    jit = pb.position_jitter_to_distribution(jitter, 2)
    coh = pb.coherence_to_distribution(energy, 0.0, 2)
    dv, dm, dpos, dw = 0.0, 0.0, 0.0, np.zeros(2)
    for (de, _, _), wc in zip(coh.samples.numpy(), coh.weights.numpy()):
        for delta, wj in zip(jit.samples.numpy(), jit.weights.numpy()):
            pj = pos + delta * (0.3 / 0.25)
            kv = 200.0 + de / 1000.0
            a, b, c = R.stem_4d_vjp(pot, 1.7, 0.25, modes, w, 0.25, kv, pj, 0.3, g * wc * wj, with_positions=True)
            dv, dm, dpos = dv + a, dm + b, dpos + c
            for k in range(2):
                per = R.stem_4d(pot, 1.7, 0.25, modes[..., k:k + 1], [1.0], 0.25, kv, pj, 0.3)["data"]
                dw[k] += wc * wj * np.sum(g * per)
    assert rel_l2(V.grad.cpu().numpy(), dv) < TOL
    assert rel_l2(md.grad.cpu().numpy(), np.conj(dm)) < TOL
    assert rel_l2(wt.grad.cpu().numpy(), dw) < TOL
    assert rel_l2(ps.grad.cpu().numpy(), dpos) < TOL


@pytest.mark.parametrize("h,w", [(32, 32), (24, 40)])
def test_ensemble_derivatives_through_tilts(h, w):
    """Reverse mode through tilted coherence samples (energy spread and angular
    divergence together), on the engine's square grid and on a rectangular any-size
    grid: the patterns against the oracle's ensemble branch (which applies the tilt
    ramp to the shifted wave), and the directional derivatives of L = sum(g * I)
    along random directions in V, the beam modes and the scan positions against
    central differences of the float64 oracle."""
    rng = np.random.default_rng(h + w)
    pot = rng.uniform(0.0, 30.0, (h, w, 2))
    probe = R.make_probe(200.0, 25.0, (h, w), 25.0, defocus_ang=-30.0)
    modes, wts = probe[..., None], np.array([1.0])
    pos = rng.uniform(-1.5, 1.5, (3, 2))
    g = rng.normal(size=(3, h, w))
    ens = pb.create_ensemble_axes(coherence=pb.coherence_to_distribution(0.4, 0.25, 2))
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(h, w))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    dev = torch.device("cuda")
    V = torch.tensor(pot, dtype=torch.float32, device=dev, requires_grad=True)
    md = torch.tensor(modes.astype(np.complex64), device=dev, requires_grad=True)
    ps = torch.tensor(pos, dtype=torch.float64, device=dev, requires_grad=True)
    det_t = dataclasses.replace(det, scan_positions_px=ps)
    s4 = pb.stem_4d(pb.PotentialSlices(V, 1.7, 0.25), pb.ProbeModes(md, torch.ones(1, device=dev), 0.25), mic,
                    det_t)
    (s4.data * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()
    beam = pb.create_probe_modes(modes, wts, 0.25)
    axes = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens, beam)]

    def loss(pot_, modes_, pos_):
        return float(np.sum(g * R.stem_4d_ensemble(pot_, 1.7, 0.25, modes_, 0.25, 200.0, pos_, 0.3, axes)))

    want = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes)
    assert rel_l2(s4.data.detach().cpu().numpy(), want) < TOL
    dV = rng.normal(size=pot.shape)
    dM = rng.normal(size=modes.shape) + 1j * rng.normal(size=modes.shape)
    dP = rng.normal(size=pos.shape)
    eps = 1e-4
    fd_v = (loss(pot + eps * dV, modes, pos) - loss(pot - eps * dV, modes, pos)) / (2 * eps)
    fd_m = (loss(pot, modes + eps * dM * np.abs(modes).max(), pos)
            - loss(pot, modes - eps * dM * np.abs(modes).max(), pos)) / (2 * eps * np.abs(modes).max())
    fd_p = (loss(pot, modes, pos + eps * dP) - loss(pot, modes, pos - eps * dP)) / (2 * eps)
    got_v = float(np.sum(V.grad.cpu().numpy() * dV))
    # torch's complex gradient is dL/d(re) + i dL/d(im): the directional derivative is Re(conj(grad) * d)
    got_m = float(np.sum(np.real(np.conj(md.grad.cpu().numpy()) * dM)))
    got_p = float(np.sum(ps.grad.cpu().numpy() * dP))
    for got, fd in [(got_v, fd_v), (got_m, fd_m), (got_p, fd_p)]:
        assert abs(got - fd) <= 2e-3 * abs(fd) + 1e-6 * abs(want).sum(), (got, fd)
    # forward mode through the same ensemble: torch.func.jvp along dV
    beam_c = pb.ProbeModes(md.detach(), torch.ones(1, device=dev), 0.25)

    def fwd(v):
        return pb.stem_4d(pb.PotentialSlices(v, 1.7, 0.25), beam_c, mic, det).data

    _, tan = torch.func.jvp(fwd, (V.detach(),), (torch.as_tensor(dV, dtype=torch.float32, device=dev),))
    got_jv = float(np.sum(g * tan.cpu().numpy()))
    assert abs(got_jv - fd_v) <= 2e-3 * abs(fd_v) + 1e-6 * abs(want).sum(), (got_jv, fd_v)


def test_ensemble_on_a_rectangular_grid():
    """Jitter and energy-spread axes on a 40 x 56 grid (the any-size path, one
    accumulating forward per energy) against the oracle's ensemble branch, with
    and without tilted coherence samples."""
    rng = np.random.default_rng(6)
    h, w, s = 40, 56, 3
    pot = rng.uniform(0.0, 40.0, (h, w, s))
    probe = R.make_probe(200.0, 25.0, (h, w), 25.0, defocus_ang=-30.0)
    modes = np.stack([probe, np.roll(probe, 2, axis=1) * (0.8 - 0.2j)], -1)
    wts = np.array([0.65, 0.35])
    pos = rng.uniform(-2, 2, (3, 2))
    ens = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(0.08, 2),
                                  coherence=pb.coherence_to_distribution(0.5, 0.0, 2))
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(h, w))
    beam = pb.create_probe_modes(modes, wts, 0.25)
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    s4 = pb.stem_4d(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic, det)
    axes = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(ens, beam)]
    want = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes)
    assert tuple(s4.data.shape) == (3, h, w)
    assert rel_l2(s4.data.cpu().numpy(), want) < TOL
    # tilted samples: the tilt folded into the first slice's potential, one call per tilt
    tilted = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(0.08, 2),
                                     coherence=pb.coherence_to_distribution(0.5, 0.2, 2))
    mic_t = pb.create_microscope_config(200.0, 25.0, ensemble=tilted, probe_shape=(h, w))
    s4t = pb.stem_4d(pb.create_potential_slices(pot, 1.7, 0.25), beam, mic_t, det)
    axes_t = [_axes_oracle(a) for a in pb.ensemble_axes_for_cbed(tilted, beam)]
    want_t = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes_t)
    assert rel_l2(s4t.data.cpu().numpy(), want_t) < TOL


def test_cbed_image_is_differentiable():
    """cbed_image under reverse mode: the engine's adjoint at the one zero position,
    against the oracle's adjoint of stem_4d there (cbed_image's unshifted beam)."""
    pot, modes, w = _setup(n=64, s=3, m=2, seed=5)
    g = np.random.default_rng(2).normal(size=(64, 64))
    dev = torch.device("cuda")
    V = torch.tensor(pot, dtype=torch.float32, device=dev, requires_grad=True)
    md = torch.tensor(modes.astype(np.complex64), device=dev, requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float32, device=dev)
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(64, 64))
    img = pb.cbed_image(pb.PotentialSlices(V, 1.7, 0.25), pb.ProbeModes(md, wt, 0.25), mic).data_array
    (img * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()
    want = R.stem_4d(pot, 1.7, 0.25, modes, w, 0.25, 200.0, np.zeros((1, 2)), 0.25)["data"][0]
    assert rel_l2(img.detach().cpu().numpy(), want) < TOL
    dv, dm = R.stem_4d_vjp(pot, 1.7, 0.25, modes, w, 0.25, 200.0, np.zeros((1, 2)), 0.25, g[None])
    assert rel_l2(V.grad.cpu().numpy(), dv) < TOL
    assert rel_l2(md.grad.cpu().numpy(), np.conj(dm)) < TOL


def test_ensemble_axis_weights_and_coherent_modes_are_differentiable():
    """Reverse mode through an explicit COHERENT probe-mode axis (its modes summed with
    its weights into one wave), an explicit jitter axis and an energy-spread axis,
    with respect to the potential and the two explicit axes' raw weights (through
    create_distribution's normalisation): directional derivatives against float64
    central differences of the oracle's ensemble branch."""
    pot, modes, w = _setup(n=32, s=2, m=2, seed=21)
    rng = np.random.default_rng(9)
    pos = rng.uniform(-1.5, 1.5, (3, 2))
    g = rng.normal(size=(3, 32, 32))
    jsmp = np.array([[0.05, -0.03], [-0.04, 0.06]])
    dev = torch.device("cuda")
    wm = torch.tensor([0.7, 0.3], dtype=torch.float64, requires_grad=True)
    wj = torch.tensor([0.45, 0.55], dtype=torch.float64, requires_grad=True)
    mode_axis = pb.create_distribution(np.arange(2.0)[:, None], wm, pb.ReductionMode.COHERENT, "probe_modes")
    jit_axis = pb.create_distribution(jsmp, wj, pb.ReductionMode.INCOHERENT, "position_jitter")
    coh = pb.coherence_to_distribution(0.4, 0.0, 2)
    ens = pb.create_ensemble_axes(probe_modes=mode_axis, position_jitter=jit_axis, coherence=coh)
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(32, 32))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    V = torch.tensor(pot, dtype=torch.float32, device=dev, requires_grad=True)
    beam = pb.ProbeModes(torch.tensor(modes.astype(np.complex64), device=dev),
                         torch.tensor(w, dtype=torch.float32, device=dev), 0.25)
    s4 = pb.stem_4d(pb.PotentialSlices(V, 1.7, 0.25), beam, mic, det)
    (s4.data * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()

    def axes_of(wm_, wj_):
        return [(np.arange(2.0)[:, None], wm_ / wm_.sum(), "coherent", "probe_modes"),
                (jsmp, wj_ / wj_.sum(), "incoherent", "position_jitter"), _axes_oracle(coh)]

    def loss(pot_, wm_, wj_):
        return float(np.sum(g * R.stem_4d_ensemble(pot_, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3,
                                                    axes_of(wm_, wj_))))

    wm0, wj0 = np.array([0.7, 0.3]), np.array([0.45, 0.55])
    want = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes_of(wm0, wj0))
    assert rel_l2(s4.data.detach().cpu().numpy(), want) < TOL
    dV, dwm, dwj = rng.normal(size=pot.shape), rng.normal(size=2), rng.normal(size=2)
    eps = 1e-5
    checks = [
        (float(np.sum(V.grad.cpu().numpy() * dV)),
         (loss(pot + eps * dV, wm0, wj0) - loss(pot - eps * dV, wm0, wj0)) / (2 * eps)),
        (float(np.sum(wm.grad.numpy() * dwm)),
         (loss(pot, wm0 + eps * dwm, wj0) - loss(pot, wm0 - eps * dwm, wj0)) / (2 * eps)),
        (float(np.sum(wj.grad.numpy() * dwj)),
         (loss(pot, wm0, wj0 + eps * dwj) - loss(pot, wm0, wj0 - eps * dwj)) / (2 * eps)),
    ]
    scale = float(np.abs(g * want).sum())
    for got, fd in checks:
        assert abs(got - fd) <= 2e-3 * abs(fd) + 1e-5 * scale, (got, fd)


@pytest.mark.parametrize("with_modes", [False, True])
def test_bind_cbed_axes_explicit_composition_matches_cbed_image(with_modes):
    """apply_distributions(axes, bind_cbed_axes(...)) against cbed_image's ensemble
    branch (the reference's test_cbed_image_ensemble_axes_match_explicit_composition,
    widened to jitter, energy and tilt, and a two-mode beam with its mode axis), and
    against the oracle's ensemble branch."""
    m = 2 if with_modes else 1
    pot, modes, w = _setup(n=32, s=2, m=m, seed=17)
    beam = pb.create_probe_modes(modes, w, 0.25)
    ens = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(0.15, 2),
                                  coherence=pb.coherence_to_distribution(0.5, 0.2, 2))
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(32, 32))
    pots = pb.create_potential_slices(pot, 1.7, 0.25)
    det = pb.create_detector_config(0.25, probe_calibration_pm=25.0)
    axes = pb.ensemble_axes_for_cbed(ens, beam)
    bound = pb.bind_cbed_axes(pots, beam, mic, det, axes)
    explicit = pb.apply_distributions(axes, bound)
    carried = pb.cbed_image(pots, beam, mic).data_array
    assert rel_l2(explicit.cpu().numpy(), carried.cpu().numpy()) < 1e-5
    want = R.ensemble_cbed(pot, 1.7, 0.25, modes, 0.25, 200.0, [_axes_oracle(a) for a in axes])
    assert rel_l2(explicit.cpu().numpy(), want) < TOL
    # the binder's contract: sample width and explicit column maps
    with pytest.raises(ValueError, match="sample width"):
        bound(torch.zeros(1, dtype=torch.float64))
    with pytest.raises(ValueError, match="column_maps"):
        pb.bind_cbed_axes(pots, beam, mic, det, axes, column_maps=("coherence",))


def test_coherent_jitter_axis_is_differentiable():
    """Reverse mode through a COHERENT jitter axis (the weighted shifts as one Fourier
    filter of the mode) with an energy-spread axis: patterns against the oracle's
    ensemble branch, and directional derivatives along V, the beam mode and the raw
    jitter weights against float64 central differences of it."""
    pot, modes, w = _setup(n=32, s=2, m=1, seed=23)
    rng = np.random.default_rng(10)
    pos = rng.uniform(-1.5, 1.5, (3, 2))
    g = rng.normal(size=(3, 32, 32))
    jsmp = np.array([[0.3, -0.2], [-0.25, 0.35], [0.1, 0.1]])
    dev = torch.device("cuda")
    wj = torch.tensor([0.5, 0.3, 0.2], dtype=torch.float64, requires_grad=True)
    jit_axis = pb.create_distribution(jsmp, wj, pb.ReductionMode.COHERENT, "position_jitter")
    coh = pb.coherence_to_distribution(0.4, 0.0, 2)
    ens = pb.create_ensemble_axes(position_jitter=jit_axis, coherence=coh)
    mic = pb.create_microscope_config(200.0, 25.0, ensemble=ens, probe_shape=(32, 32))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    V = torch.tensor(pot, dtype=torch.float32, device=dev, requires_grad=True)
    md = torch.tensor(modes.astype(np.complex64), device=dev, requires_grad=True)
    beam = pb.ProbeModes(md, torch.ones(1, dtype=torch.float32, device=dev), 0.25)
    s4 = pb.stem_4d(pb.PotentialSlices(V, 1.7, 0.25), beam, mic, det)
    (s4.data * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()

    def axes_of(wj_):
        return [(jsmp, wj_ / wj_.sum(), "coherent", "position_jitter"), _axes_oracle(coh)]

    def loss(pot_, modes_, wj_):
        return float(np.sum(g * R.stem_4d_ensemble(pot_, 1.7, 0.25, modes_, 0.25, 200.0, pos, 0.3, axes_of(wj_))))

    wj0 = np.array([0.5, 0.3, 0.2])
    want = R.stem_4d_ensemble(pot, 1.7, 0.25, modes, 0.25, 200.0, pos, 0.3, axes_of(wj0))
    assert rel_l2(s4.data.detach().cpu().numpy(), want) < TOL
    dV, dwj = rng.normal(size=pot.shape), rng.normal(size=3)
    dM = (rng.normal(size=modes.shape) + 1j * rng.normal(size=modes.shape)) * np.abs(modes).max()
    eps = 1e-5
    checks = [
        (float(np.sum(V.grad.cpu().numpy() * dV)),
         (loss(pot + eps * dV, modes, wj0) - loss(pot - eps * dV, modes, wj0)) / (2 * eps)),
        (float(np.sum(np.real(np.conj(md.grad.cpu().numpy()) * dM))),
         (loss(pot, modes + eps * dM, wj0) - loss(pot, modes - eps * dM, wj0)) / (2 * eps)),
        (float(np.sum(wj.grad.numpy() * dwj)),
         (loss(pot, modes, wj0 + eps * dwj) - loss(pot, modes, wj0 - eps * dwj)) / (2 * eps)),
    ]
    scale = float(np.abs(g * want).sum())
    for got, fd in checks:
        assert abs(got - fd) <= 2e-3 * abs(fd) + 1e-5 * scale, (got, fd)
