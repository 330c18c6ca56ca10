"""Virtual detectors on the GPU: standalone integration and the fused pattern-pass
epilogue, against the oracle's annular_detector."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_annular_detector_known_answer():
    """test_simulations.py:84-122."""
    data = torch.arange(6 * 4 * 4, dtype=torch.float32).reshape(6, 4, 4).cuda()
    s4 = pb.create_stem4d(data, 0.5, 0.25, np.zeros((6, 2)), 80.0)
    det = pb.create_detector_config(0.5, collection_inner_mrad=0.0, collection_outer_mrad=1000.0, scan_shape=(2, 3))
    img = pb.annular_detector(s4, det)
    assert img.real_space and img.calib_y == 0.5
    assert np.array_equal(img.data_array.cpu().numpy(), [[120.0, 376.0, 632.0], [888.0, 1144.0, 1400.0]])


def test_annular_detector_matches_oracle_on_golden(golden):
    g = golden
    data = torch.from_numpy(g["stem4d"].astype(np.float32)).cuda()
    fc = 1.0 / (32 * 0.2)
    s4 = pb.create_stem4d(data, 0.2, fc, g["positions_px"] * 0.2, 100.0)
    for inner, outer in [(0.0, 1e6), (0.0, 10.0), (10.0, 25.0), (25.0, 60.0)]:
        det = pb.create_detector_config(0.2, collection_inner_mrad=inner, collection_outer_mrad=outer,
                                        scan_shape=(2, 2))
        got = pb.annular_detector(s4, det).data_array.cpu().numpy()
        want = R.annular_detector(g["stem4d"].astype(np.float32), fc, 100.0, inner, outer, (2, 2))
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


def _case(n, S, M, P, seed, kv=200.0, calib=0.2):
    rng = np.random.default_rng(seed)
    pot = rng.uniform(0, 20, (n, n, S))
    probe = R.make_probe(kv, 25.0, (n, n), calib * 100.0, defocus_ang=-30.0)
    modes = np.stack([probe * (1.0 if m == 0 else 0.6) * np.exp(1j * m) for m in range(M)], axis=-1)
    w = np.linspace(1.0, 0.5, M)
    w = w / w.sum()
    pos = rng.uniform(-3, 3, (P, 2))
    return pot, modes, w, pos


@pytest.mark.parametrize("n,S,M", [(16, 3, 1), (64, 4, 2), (128, 5, 1), (256, 2, 1)])
def test_fused_detectors_match_oracle(n, S, M):
    P, calib, kv = 12, 0.2, 200.0
    pot, modes, w, pos = _case(n, S, M, P, n + S)
    annuli = [(0.0, 12.0), (12.0, 25.0), (30.0, 90.0), (0.0, 1e6)]
    pots = pb.create_potential_slices(pot, 1.5, calib)
    beam = pb.create_probe_modes(modes, w, calib)
    mic = pb.create_microscope_config(kv, 25.0, probe_shape=(n, n))
    det = pb.create_detector_config(calib, scan_positions_px=pos, scan_shape=(3, 4))
    got = pb.stem_4d_detectors(pots, beam, mic, det, annuli).cpu().numpy()
    pats = R.stem_4d(pot, 1.5, calib, modes, w, calib, kv, pos, calib, dtype=np.complex128)["data"]
    fc = 1.0 / (n * calib)
    for d, (a, b) in enumerate(annuli):
        want = R.annular_detector(pats, fc, kv, a, b, (P,))
        assert rel_l2(got[:, d], want) < 1e-5, (d, a, b)
    # the full-field detector collects the aperture count of every mode
    assert np.allclose(got[:, 3], got[0, 3], rtol=1e-5)


def test_fused_equals_unfused_and_keeps_patterns():
    n, S, P, calib, kv = 128, 6, 64, 0.2, 200.0
    pot, modes, w, pos = _case(n, S, 1, P, 3)
    pots = pb.create_potential_slices(pot, 1.5, calib)
    beam = pb.create_probe_modes(modes, w, calib)
    mic = pb.create_microscope_config(kv, 25.0, probe_shape=(n, n))
    det = pb.create_detector_config(calib, collection_inner_mrad=30.0, collection_outer_mrad=80.0,
                                    scan_positions_px=pos, scan_shape=(8, 8))
    s4 = pb.stem_4d(pots, beam, mic, det)
    unfused = pb.annular_detector(s4, det).data_array
    fused = pb.stem_4d_annular(pots, beam, mic, det).data_array
    assert fused.shape == (8, 8) and fused.dtype == torch.float64
    assert torch.allclose(fused, unfused, rtol=1e-5, atol=1e-9)
    # patterns stored alongside the detector sums are the plain forward's patterns
    from ptyrodactyl_b200.detectors import detector_mask_bits, run_forward_detect
    dev = torch.device("cuda")
    sl = torch.as_tensor(pot, dtype=torch.float32, device=dev)
    md = torch.as_tensor(modes, dtype=torch.complex64, device=dev)
    wt = torch.as_tensor(w, dtype=torch.float32, device=dev)
    ps = torch.as_tensor(pos, dtype=torch.float64, device=dev)
    mask = detector_mask_bits(n, 1.0 / (n * calib), kv, [(30.0, 80.0)], dev)
    pats = torch.empty((P, n, n), dtype=torch.float32, device=dev)
    vals = run_forward_detect(sl, 1.5, md, wt, ps, kv, calib, calib, mask, 1, patterns=pats)
    assert torch.equal(pats, s4.data)
    assert torch.allclose(vals[:, 0].reshape(8, 8), unfused, rtol=1e-5, atol=1e-9)
    # accumulate adds the detector sums of a second configuration
    acc = vals.clone()
    run_forward_detect(sl, 1.5, md, wt, ps, kv, calib, calib, mask, 1, out=acc, accumulate=True)
    assert torch.allclose(acc, 2 * vals, rtol=1e-12)


def test_detector_argument_errors():
    data = torch.zeros((4, 8, 8), device="cuda")
    s4 = pb.create_stem4d(data, 0.5, 0.25, np.zeros((4, 2)), 80.0)
    with pytest.raises(ValueError, match="scan_shape is required"):
        pb.annular_detector(s4, pb.create_detector_config(0.5))
    with pytest.raises(ValueError, match="between 1 and 32"):
        pb.virtual_detectors(s4, [(0.0, 1.0)] * 33)
    with pytest.raises(ValueError, match="inner <= outer"):
        pb.virtual_detectors(s4, [(2.0, 1.0)])


@pytest.mark.parametrize("shape,extent,out", [((128, 128), 30.0, (64, 64)), ((256, 256), 45.0, (100, 80)),
                                              ((64, 64), 10.0, (48, 48)), ((128, 128), 500.0, (128, 128))])
def test_clip_cbed_matches_oracle(shape, extent, out):
    rng = np.random.default_rng(shape[0] + int(extent))
    pats = rng.uniform(0, 1, (5,) + shape)
    fc = 1.0 / (shape[0] * 0.2)
    got = pb.clip_cbed(torch.as_tensor(pats, dtype=torch.float32, device="cuda"), fc, 200.0, extent, out)
    want = np.stack([R.clip_cbed(p, fc, 200.0, extent, out) for p in pats])
    assert got.shape == want.shape
    assert rel_l2(got.cpu().numpy(), want) < 1e-6
    one = pb.clip_cbed(torch.as_tensor(pats[0], dtype=torch.float32, device="cuda"), fc, 200.0, extent, out)
    assert torch.allclose(one, got[0])


def test_stem_4d_clipped_matches_clipped_stem_4d():
    n, S, P, calib, kv = 128, 3, 9, 0.2, 200.0
    pot, modes, w, pos = _case(n, S, 1, P, 5)
    pots = pb.create_potential_slices(pot, 1.5, calib)
    beam = pb.create_probe_modes(modes, w, calib)
    mic = pb.create_microscope_config(kv, 25.0, probe_shape=(n, n))
    det = pb.create_detector_config(calib, scan_positions_px=pos)
    full = pb.stem_4d(pots, beam, mic, det)
    clipped = pb.stem_4d_clipped(pots, beam, mic, det, 40.0, (64, 64), chunk=4)
    want = pb.clip_cbed(full.data, full.fourier_space_calib, kv, 40.0, (64, 64))
    assert torch.equal(clipped.data, want)
    lam = R.relativistic_wavelength_ang(kv)
    assert abs(clipped.fourier_space_calib - (80.0 / 64) / (lam * 1000.0)) < 1e-15


@pytest.mark.parametrize("shape", [(48, 80), (33, 33), (7, 5), (64, 64)])
def test_virtual_detectors_any_pattern_shape(shape):
    """annular_detector at any (H, W), odd and rectangular, as the reference integrates
    any pattern shape (simulations.py:1600-1636)."""
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    pats = rng.uniform(0.0, 1.0, (6,) + shape).astype(np.float32)
    fc, kv = 0.05, 200.0
    s4 = pb.create_stem4d(torch.from_numpy(pats).cuda(), 0.3, fc, np.zeros((6, 2)), kv)
    annuli = [(0.0, 5.0), (5.0, 12.0), (12.0, 40.0), (0.0, 1e6)]
    got = pb.virtual_detectors(s4, annuli).cpu().numpy()
    for d, (a, b) in enumerate(annuli):
        want = R.annular_detector(pats, fc, kv, a, b, (6,))
        assert np.allclose(got[:, d], want, rtol=1e-12, atol=1e-9), (shape, d)
    det = pb.create_detector_config(0.3, collection_inner_mrad=5.0, collection_outer_mrad=12.0, scan_shape=(2, 3))
    img = pb.annular_detector(s4, det).data_array.cpu().numpy()
    assert np.allclose(img, R.annular_detector(pats, fc, kv, 5.0, 12.0, (2, 3)), rtol=1e-12, atol=1e-9)


def test_detectors_on_any_size_grid_and_with_ensemble():
    """stem_4d_detectors where the fused epilogue does not apply (an any-size grid; an
    ensemble microscope): stem_4d's own path, then the masked sums, equal to
    annular_detector(stem_4d(...))."""
    calib, kv = 0.25, 200.0
    annuli = [(0.0, 12.0), (12.0, 40.0)]
    rng = np.random.default_rng(5)
    # any-size grid: 40 x 56
    h, w = 40, 56
    pot = rng.uniform(0.0, 20.0, (h, w, 3))
    probe = R.make_probe(kv, 25.0, (h, w), calib * 100.0, defocus_ang=-30.0)
    pos = rng.uniform(-2, 2, (5, 2))
    pots = pb.create_potential_slices(pot, 1.5, calib)
    beam = pb.create_probe_modes(probe[..., None], np.array([1.0]), calib)
    mic = pb.create_microscope_config(kv, 25.0, probe_shape=(h, w))
    det = pb.create_detector_config(calib, scan_positions_px=pos, scan_shape=(5, 1))
    got = pb.stem_4d_detectors(pots, beam, mic, det, annuli).cpu().numpy()
    pats = R.stem_4d(pot, 1.5, calib, probe[..., None], np.array([1.0]), calib, kv, pos, calib,
                     dtype=np.complex128)["data"]
    for d, (a, b) in enumerate(annuli):
        assert rel_l2(got[:, d], R.annular_detector(pats, 1.0 / (h * calib), kv, a, b, (5,))) < 1e-5
    # ensemble axes on the engine grid
    n = 64
    pot = rng.uniform(0.0, 20.0, (n, n, 3))
    probe = R.make_probe(kv, 25.0, (n, n), calib * 100.0, defocus_ang=-30.0)
    ens = pb.create_ensemble_axes(position_jitter=pb.position_jitter_to_distribution(0.08, 2),
                                  coherence=pb.coherence_to_distribution(0.5, 0.0, 2))
    mic = pb.create_microscope_config(kv, 25.0, ensemble=ens, probe_shape=(n, n))
    pots = pb.create_potential_slices(pot, 1.5, calib)
    beam = pb.create_probe_modes(probe[..., None], np.array([1.0]), calib)
    det = pb.create_detector_config(calib, collection_inner_mrad=12.0, collection_outer_mrad=40.0,
                                    scan_positions_px=pos, scan_shape=(5, 1))
    fused = pb.stem_4d_annular(pots, beam, mic, det).data_array
    unfused = pb.annular_detector(pb.stem_4d(pots, beam, mic, det), det).data_array
    assert torch.allclose(fused, unfused, rtol=1e-12, atol=0.0)
