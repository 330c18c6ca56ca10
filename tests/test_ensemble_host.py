"""Host logic of the ensemble path (no GPU): the beam tilt folded into the first
slice's potential equals the reference's tilt ramp applied to the wave."""

import numpy as np
import torch

from oracle import multislice_ref as R
from ptyrodactyl_b200.ensemble import tilt_folded_slices
from ptyrodactyl_b200.simulations import interaction_sigma


def test_tilt_fold_is_the_tilt_ramp():
    """exp(i sigma V_0') == exp(i sigma V_0) * ramp, to the float32 rounding of V_0'
    (|V_0'| <= max V + pi / sigma), for square and rectangular grids."""
    rng = np.random.default_rng(0)
    for (h, w), tilt, kv, calib in [((32, 32), (0.3, -0.2), 200.0, 0.25), ((24, 40), (-1.5, 0.7), 80.0, 0.1),
                                    ((7, 5), (4.0, 2.0), 300.0, 0.4)]:
        pot = rng.uniform(0.0, 30.0, (h, w, 3)).astype(np.float32)
        folded = tilt_folded_slices(torch.from_numpy(pot), tilt, kv, calib).numpy()
        assert folded.shape == pot.shape and folded.dtype == np.float32
        assert np.array_equal(folded[:, :, 1:], pot[:, :, 1:])
        sigma = interaction_sigma(kv)
        got = np.exp(1j * sigma * folded[:, :, 0].astype(np.float64))
        want = np.exp(1j * sigma * pot[:, :, 0].astype(np.float64))[..., None]
        want = R.tilt_phase_ramp(want, np.asarray(tilt), kv, calib)[..., 0]
        bound = sigma * np.spacing(np.float32(np.abs(folded[:, :, 0]).max()))
        assert np.max(np.abs(got - want)) <= bound + 1e-12


def test_tilt_fold_passes_the_potential_gradient():
    pot = torch.rand(6, 8, 2, dtype=torch.float32, requires_grad=True)
    folded = tilt_folded_slices(pot, (0.5, 0.5), 200.0, 0.2)
    g = torch.randn_like(folded)
    (folded * g).sum().backward()
    assert torch.equal(pot.grad, g)


def test_axis_samples_read_inside_torch_func_transforms():
    """The ensemble's constant sample tables are read on the host also under
    torch.func.jvp, where a plain .detach().numpy() has no storage to read."""
    from ptyrodactyl_b200.ensemble import _host
    s = torch.tensor([1.0, 2.0])
    out, tan = torch.func.jvp(lambda x: x * float(_host(s).sum()), (torch.ones(2),), (torch.ones(2),))
    assert torch.equal(out, torch.full((2,), 3.0)) and torch.equal(tan, torch.full((2,), 3.0))
