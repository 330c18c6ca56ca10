"""GPU parity of the any-size path (ptyro_gm_*): every height x width in [1, 4096]
that is not one of the pass engine's square power-of-two grids.

The reference's stem_4d, its jax.grad and make_probe take any probe_shape
(multislice/simulations.py:334-431, 1330-1443); the oracle restates them for any
shape. The any-size transforms are direct four-step DFTs in float32, so the tolerance
is the gradient tests' relative L2 of 1e-4 against the complex128 oracle, with
1e-5 for the probe and the plain transforms.
"""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4
TOL_FFT = 1e-5
DZ, KV, CALIB = 1.7, 200.0, 0.3


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _case(h, w, s, m, p, seed=0):
    rng = np.random.default_rng(seed)
    pot = rng.uniform(0.0, 60.0, (h, w, s))
    probe = R.make_probe(KV, 25.0, (h, w), 30.0, defocus_ang=-20.0, c3_ang=1e-3)
    # a little noise keeps every pixel of the tiny grids lit
    probe = probe + 0.05 * np.abs(probe).max(initial=1.0) * (rng.normal(size=(h, w)) + 1j * rng.normal(size=(h, w)))
    modes = probe[..., None]
    if m == 2:
        modes = np.stack([probe, np.roll(probe, 1, axis=1) * (0.7 - 0.3j)], axis=-1)
    wt = np.array([1.0]) if m == 1 else np.array([0.6, 0.4])
    pos = rng.uniform(-3, 3, (p, 2))
    g = rng.normal(size=(p, h, w))
    return pot, modes, wt, pos, g


def _dev(*arrays):
    dev = torch.device("cuda")
    out = []
    for a in arrays:
        if np.iscomplexobj(a):
            out.append(torch.as_tensor(a.astype(np.complex64), device=dev))
        elif a.dtype == np.float64 and a.ndim == 2 and a.shape[1] == 2:
            out.append(torch.as_tensor(a, dtype=torch.float64, device=dev))
        else:
            out.append(torch.as_tensor(a, dtype=torch.float32, device=dev))
    return out


SHAPES = [(96, 160, 4, 2, 3), (45, 77, 3, 1, 2), (31, 37, 2, 1, 2), (3, 5, 2, 2, 2), (100, 100, 3, 1, 2),
          (64, 128, 3, 1, 2), (4, 4, 1, 2, 2), (8, 1021, 2, 1, 2), (1, 64, 2, 1, 2), (4, 3000, 2, 1, 2),
          (4096, 3, 2, 1, 1), (384, 640, 2, 1, 2)]


@pytest.mark.parametrize("h,w,s,m,p", SHAPES)
def test_forward_matches_oracle(h, w, s, m, p):
    pot, modes, wt, pos, _ = _case(h, w, s, m, p, seed=h * 7 + w)
    sl, md, ww = _dev(pot, modes, wt)
    ps = torch.as_tensor(pos, dtype=torch.float64, device="cuda")
    status = pb._lib.new_status(sl.device)
    out = pb.simulations.run_forward(sl, DZ, md, ww, ps, KV, CALIB, CALIB, status=status)
    pb._lib.check_status(status, "any-size forward")
    assert tuple(out.shape) == (p, h, w)
    want = R.stem_4d(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB)["data"]
    assert rel_l2(out.cpu().numpy(), want) < TOL, rel_l2(out.cpu().numpy(), want)


def test_forward_batches_and_accumulate_agree():
    h, w = 40, 56
    pot, modes, wt, pos, _ = _case(h, w, 3, 2, 7, seed=5)
    sl, md, ww = _dev(pot, modes, wt)
    ps = torch.as_tensor(pos, dtype=torch.float64, device="cuda")
    a = pb.simulations.run_forward(sl, DZ, md, ww, ps, KV, CALIB, CALIB)
    b = pb.simulations.run_forward(sl, DZ, md, ww, ps, KV, CALIB, CALIB, batch=2)
    assert torch.equal(a, b)
    acc = a.clone()
    pb.simulations.run_forward(sl, DZ, md, ww, ps, KV, CALIB, CALIB, out=acc, accumulate=True, batch=3)
    assert torch.allclose(acc, 2 * a, rtol=1e-6, atol=0)


@pytest.mark.parametrize("h,w,s,m,p", [(48, 80, 3, 2, 3), (33, 27, 2, 1, 2), (64, 128, 2, 1, 2), (5, 7, 2, 1, 3),
                                       (4, 4, 2, 2, 2)])
def test_vjp_matches_oracle(h, w, s, m, p):
    pot, modes, wt, pos, g = _case(h, w, s, m, p, seed=h + w)
    sl, md, ww, gg = _dev(pot, modes, wt, g)
    ps = torch.as_tensor(pos, dtype=torch.float64, device="cuda")
    out, dv, dm = pb.vjp(sl, md, ww, ps, gg, DZ, KV, CALIB)
    dv_ref, dm_ref = R.stem_4d_vjp(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB, g)
    want = R.stem_4d(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB)["data"]
    assert rel_l2(out.cpu().numpy(), want) < TOL
    assert rel_l2(dv.cpu().numpy(), dv_ref) < TOL, rel_l2(dv.cpu().numpy(), dv_ref)
    assert rel_l2(dm.cpu().numpy(), dm_ref) < TOL, rel_l2(dm.cpu().numpy(), dm_ref)


@pytest.mark.parametrize("h,w,s,m,p", [(48, 80, 3, 2, 3), (33, 27, 2, 1, 2)])
def test_autograd_position_and_weight_gradients(h, w, s, m, p):
    pot, modes, wt, pos, g = _case(h, w, s, m, p, seed=3 * h + w)
    sl, md, gg = _dev(pot, modes, g)
    sl.requires_grad_(True)
    md.requires_grad_(True)
    ww = torch.as_tensor(wt, dtype=torch.float32, device="cuda").requires_grad_(True)
    ps = torch.as_tensor(pos, dtype=torch.float64, device="cuda").requires_grad_(True)
    pat = pb.stem_4d_patterns(sl, md, ww, ps, DZ, KV, CALIB)
    (pat * gg).sum().backward()
    dv_ref, dm_ref, dpos = R.stem_4d_vjp(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB, g, with_positions=True)
    assert rel_l2(sl.grad.cpu().numpy(), dv_ref) < TOL
    # torch's convention 2 dL/dconj(z) is the conjugate of JAX's
    assert rel_l2(md.grad.cpu().numpy(), np.conj(dm_ref)) < TOL
    assert rel_l2(ps.grad.cpu().numpy(), dpos) < TOL, rel_l2(ps.grad.cpu().numpy(), dpos)
    per_mode = [R.stem_4d(pot, DZ, CALIB, modes[..., k:k + 1], [1.0], CALIB, KV, pos, CALIB)["data"]
                for k in range(m)]
    want_w = np.array([np.sum(g * per_mode[k]) for k in range(m)])
    assert rel_l2(ww.grad.cpu().numpy(), want_w) < TOL


@pytest.mark.parametrize("h,w,s,m,p", [(48, 80, 3, 2, 3), (33, 27, 2, 1, 2), (4, 4, 2, 1, 2)])
def test_forward_mode_matches_oracle(h, w, s, m, p):
    """ptyro_gm_jvp against the oracle's stem_4d_jvp for potential and mode tangents,
    directly and through torch.func.jvp of the public differentiable forward."""
    pot, modes, wt, pos, _ = _case(h, w, s, m, p, seed=5 * h + w)
    rng = np.random.default_rng(h * w)
    dpot = rng.normal(size=pot.shape)
    dmodes = 0.1 * (rng.normal(size=modes.shape) + 1j * rng.normal(size=modes.shape))
    sl, md, ww, dsl, dmd = _dev(pot, modes, wt, dpot, dmodes)
    ps = torch.as_tensor(pos, dtype=torch.float64, device="cuda")
    want, dwant = R.stem_4d_jvp(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB, dslices=dpot, dbeam=dmodes)
    out, tan = pb.jvp(sl, md, ww, ps, dsl, dmd, DZ, KV, CALIB)
    assert rel_l2(out.cpu().numpy(), want) < TOL
    assert rel_l2(tan.cpu().numpy(), dwant) < TOL, rel_l2(tan.cpu().numpy(), dwant)
    _, tan_v = pb.jvp(sl, md, ww, ps, dsl, None, DZ, KV, CALIB, want_patterns=False)
    _, dwant_v = R.stem_4d_jvp(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB, dslices=dpot)
    assert rel_l2(tan_v.cpu().numpy(), dwant_v) < TOL
    _, tan_f = torch.func.jvp(lambda v, b: pb.stem_4d_patterns(v, b, ww, ps, DZ, KV, CALIB), (sl, md), (dsl, dmd))
    assert rel_l2(tan_f.cpu().numpy(), dwant) < TOL


@pytest.mark.parametrize("h,w", [(96, 160), (45, 77), (64, 128), (7, 5), (100, 100)])
def test_make_probe_matches_oracle(h, w):
    mic = pb.create_microscope_config(KV, 25.0, probe_shape=(h, w), defocus_ang=-35.0, c3_ang=2e-3)
    det = pb.create_detector_config(0.3, 30.0)
    got = pb.make_probe(mic, det).cpu().numpy()
    want = R.make_probe(KV, 25.0, (h, w), 30.0, defocus_ang=-35.0, c3_ang=2e-3)
    assert got.shape == (h, w)
    assert rel_l2(got, want) < TOL_FFT, rel_l2(got, want)
    diff = pb.make_probe_differentiable(KV, 25.0, (h, w), 30.0, -35.0, 2e-3).detach().cpu().numpy()
    assert rel_l2(diff, want) < TOL_FFT, rel_l2(diff, want)


@pytest.mark.parametrize("h,w", [(45, 77), (1, 9), (12, 30), (210, 7)])
def test_fft2_matches_numpy(h, w):
    rng = np.random.default_rng(h * w)
    x = rng.normal(size=(3, h, w)) + 1j * rng.normal(size=(3, h, w))
    xt = torch.as_tensor(x.astype(np.complex64), device="cuda")
    assert rel_l2(pb.simulations.fft2(xt).cpu().numpy(), np.fft.fft2(x)) < TOL_FFT
    assert rel_l2(pb.simulations.fft2(xt, inverse=True).cpu().numpy(), np.fft.ifft2(x)) < TOL_FFT


def test_public_stem_4d_and_cbed_on_a_rectangular_grid():
    h, w, s = 40, 56, 3
    pot, modes, wt, pos, _ = _case(h, w, s, 1, 4, seed=9)
    mic = pb.create_microscope_config(KV, 25.0, probe_shape=(h, w))
    det = pb.create_detector_config(CALIB, 30.0, scan_positions_px=pos)
    beam = pb.create_probe_modes(modes, wt, CALIB)
    slices = pb.create_potential_slices(torch.as_tensor(pot, dtype=torch.float32, device="cuda"), DZ, CALIB)
    s4 = pb.stem_4d(slices, beam, mic, det)
    want = R.stem_4d(pot, DZ, CALIB, modes, wt, CALIB, KV, pos, CALIB)
    assert tuple(s4.data.shape) == (4, h, w)
    assert rel_l2(s4.data.cpu().numpy(), want["data"]) < TOL
    assert abs(float(s4.fourier_space_calib) - want["fourier_space_calib"]) < 1e-12
    host = torch.empty((4, h, w), dtype=torch.float32).pin_memory()
    pb.stem_4d(slices, beam, mic, det, out=host)
    assert torch.equal(host, s4.data.cpu())
    amp = pb.simulations.cbed_amplitude(slices, beam, mic).cpu().numpy()
    want_amp = R.cbed_amplitude(pot, DZ, KV, CALIB, modes)
    assert rel_l2(amp, want_amp) < TOL
    img = pb.cbed_image(slices, beam, mic)
    want_img = R.cbed_image(pot, DZ, CALIB, modes, wt, CALIB, KV)
    assert rel_l2(img.data_array.cpu().numpy(), want_img) < TOL


def test_windows_are_refused_off_the_engine_grids():
    pot, modes, wt, pos, _ = _case(24, 40, 2, 1, 2)
    sl, md, ww = _dev(pot, modes, wt)
    ps = torch.as_tensor(pos, dtype=torch.float64, device="cuda")
    win = torch.zeros((2, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError, match="windows"):
        pb.simulations.run_forward(sl, DZ, md, ww, ps, KV, CALIB, CALIB, windows=win)
