"""Validated entry points: structure errors (ValueError) and value errors
(CheckedValueError, a RuntimeError) with the reference's messages, raised before
any GPU work (checked.py)."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from ptyrodactyl_b200.checked import CheckedValueError


def _inputs(n=16):
    pots = pb.PotentialSlices(torch.zeros((n, n, 2)), 1.0, 0.5)
    beam = pb.ProbeModes(torch.ones((n, n, 1), dtype=torch.complex64), torch.ones(1), 0.5)
    mic = pb.create_microscope_config(80.0, 20.0, probe_shape=(n, n))
    det = pb.create_detector_config(0.5, scan_positions_px=[[1.0, 2.0], [3.0, 4.0]])
    return pots, beam, mic, det


def test_structure_errors():
    pots, beam, mic, det = _inputs()
    bad_beam = pb.ProbeModes(torch.ones((8, 8, 1), dtype=torch.complex64), torch.ones(1), 0.5)
    with pytest.raises(ValueError, match="beam.modes spatial shape must match pot_slice.slices"):
        pb.checked_stem_4d(pots, bad_beam, mic, det)
    with pytest.raises(ValueError, match="beam.weights must have shape"):
        pb.checked_stem_4d(pots, pb.ProbeModes(beam.modes, torch.ones(2), 0.5), mic, det)
    with pytest.raises(ValueError, match="detector.scan_positions_px is required"):
        pb.checked_stem_4d(pots, beam, mic, pb.create_detector_config(0.5))
    with pytest.raises(ValueError, match="microscope.probe_shape is required"):
        pb.checked_make_probe(pb.create_microscope_config(80.0, 20.0), det)


def test_value_errors():
    pots, beam, mic, det = _inputs()
    nan_pots = pb.PotentialSlices(torch.full((16, 16, 2), float("nan")), 1.0, 0.5)
    with pytest.raises(CheckedValueError, match="pot_slice.slices contain non-finite values"):
        pb.checked_stem_4d(nan_pots, beam, mic, det)
    far = pb.create_detector_config(0.5, scan_positions_px=[[1.0, 2.0], [30.0, 4.0]])
    with pytest.raises(CheckedValueError, match="positions must be within pot_slice grid bounds"):
        pb.checked_stem_4d(pots, beam, mic, far)
    neg = pb.PotentialSlices(pots.slices, -1.0, 0.5)
    with pytest.raises(CheckedValueError, match="pot_slice.slice_thickness must be positive"):
        pb.checked_stem_4d(neg, beam, mic, det)
    assert issubclass(CheckedValueError, RuntimeError)


def test_sharded_checks():
    pots, beam, mic, _ = _inputs()
    sample = pb.create_atomic_slice_data(np.zeros((2, 3)), [0, 0], [[0.0, 1.0]], np.zeros((1, 16, 16)))
    with pytest.raises(ValueError, match="detector.scan_positions_ang is required"):
        pb.checked_stem4d_sharded(beam, sample, mic, pb.create_detector_config(0.5))
    out_of_grid = pb.create_detector_config(0.5, scan_positions_ang=[[1.0, 9.0]])
    with pytest.raises(CheckedValueError, match="within atom_potentials grid bounds"):
        pb.checked_stem4d_sharded(beam, sample, mic, out_of_grid)


@pytest.mark.gpu
def test_checked_entries_match_unchecked_on_valid_inputs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(5)
    n = 64
    pots = pb.create_potential_slices(torch.as_tensor(rng.uniform(0, 30, (n, n, 3)), dtype=torch.float32), 1.5, 0.2)
    mic = pb.create_microscope_config(200.0, 25.0, 10.0, probe_shape=(n, n))
    det = pb.create_detector_config(0.2, scan_positions_px=rng.uniform(0, n - 1, (9, 2)))
    probe = pb.checked_make_probe(mic, det)
    assert torch.equal(probe.cpu(), pb.make_probe(mic, det).cpu())
    beam = pb.create_probe_modes(probe.cpu().numpy()[..., None], [1.0], 0.2)
    got = pb.checked_stem_4d(pots, beam, mic, det).data.cpu()
    assert torch.equal(got, pb.stem_4d(pots, beam, mic, det).data.cpu())
    cb = pb.checked_cbed_image(pots, beam, mic)
    assert torch.equal(cb.data_array.cpu(), pb.cbed_image(pots, beam, mic).data_array.cpu())
    sample = pb.create_atomic_slice_data(np.array([[2.0, 2.5, 0.25], [4.5, 5.0, 1.25]]), [0, 0],
                                         [[0.0, 1.0], [1.0, 2.0]], rng.uniform(0, 1, (1, n, n)))
    det_ang = pb.create_detector_config(0.2, scan_positions_ang=rng.uniform(0, n * 0.2 - 0.5, (5, 2)))
    got = pb.checked_stem4d_sharded(beam, sample, mic, det_ang).data.cpu()
    assert torch.equal(got, pb.stem4d_sharded(beam, sample, mic, det_ang).data.cpu())


def test_public_integrator_signatures_have_at_most_six_parameters():
    """The reference's contract on its public integrators (test_simulations.py:59-81)."""
    import inspect
    for f in (pb.aberration, pb.annular_detector, pb.cbed_amplitude, pb.cbed_image, pb.checked_cbed_image,
              pb.checked_make_probe, pb.checked_stem4d_sharded, pb.checked_stem_4d, pb.make_probe,
              pb.stem4d_sharded, pb.stem_4d):
        assert len(inspect.signature(f).parameters) <= 6, f


def test_aberration_matches_oracle_and_differentiates():
    import numpy as np
    import torch
    from oracle import multislice_ref as R
    q = np.linspace(0.0, 1.2, 50).reshape(5, 10)
    lam = R.relativistic_wavelength_ang(200.0)
    want = R.aberration(q, lam, -35.0, 2e-3, 0.5)
    got = pb.aberration(q, lam, -35.0, 2e-3, 0.5)
    assert got.dtype == torch.float64 and np.allclose(got.numpy(), want, rtol=1e-14, atol=1e-12)
    c1 = torch.tensor(-35.0, dtype=torch.float64, requires_grad=True)
    pb.aberration(torch.as_tensor(q), lam, c1).sum().backward()
    assert abs(float(c1.grad) - float(np.sum(2 * np.pi / lam * (lam * q) ** 2 / 2))) < 1e-9 * abs(float(c1.grad))
