"""GPU parity of the adjoint kernels (the ptychographic gradient).

The reference gradient is jax.grad through stem_4d; the oracle restates it by
hand (oracle/multislice_ref.py: stem_4d_vjp), itself checked against central
finite differences on the CPU (tests/test_oracle.py). Tolerance: relative L2
<= 1e-4 against the complex128 oracle for dL/dV and dL/dbeam.
"""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from ptyrodactyl_b200 import synth
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _case(n=64, s=5, m=1, p=3, seed=0):
    rng = np.random.default_rng(seed)
    pot = rng.uniform(0.0, 60.0, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0, c3_ang=1e-3)
    modes = probe[..., None]
    if m == 2:
        modes = np.stack([probe, np.roll(probe, 2, axis=1) * (0.7 - 0.3j)], axis=-1)
    w = np.array([1.0]) if m == 1 else np.array([0.6, 0.4])
    pos = rng.uniform(-3, 3, (p, 2))
    g = rng.normal(size=(p, n, n))
    return pot, modes, w, pos, g


def _gpu_vjp(pot, modes, w, pos, g, dz=1.7, kv=200.0, calib=0.3, ckpt=0, batch=0):
    dev = torch.device("cuda")
    out, dv, dm = pb.vjp(torch.as_tensor(pot, dtype=torch.float32, device=dev),
                         torch.as_tensor(modes.astype(np.complex64), device=dev),
                         torch.as_tensor(w, dtype=torch.float32, device=dev),
                         torch.as_tensor(pos, dtype=torch.float64, device=dev),
                         torch.as_tensor(g, dtype=torch.float32, device=dev), dz, kv, calib,
                         ckpt_every=ckpt, batch=batch)
    torch.cuda.synchronize()
    return out.cpu().numpy(), dv.cpu().numpy(), dm.cpu().numpy()


@pytest.mark.parametrize("n,s,m,p,ckpt", [(64, 5, 1, 3, 0), (64, 4, 2, 2, 1), (128, 7, 1, 2, 3), (256, 3, 1, 2, 0),
                                          (32, 1, 1, 3, 0)])
def test_vjp_matches_oracle(n, s, m, p, ckpt):
    pot, modes, w, pos, g = _case(n, s, m, p)
    out, dv, dm = _gpu_vjp(pot, modes, w, pos, g, ckpt=ckpt)
    want_out = R.stem_4d(pot, 1.7, 0.3, modes, w, 0.3, 200.0, pos, 0.3)["data"]
    dv_ref, dm_ref = R.stem_4d_vjp(pot, 1.7, 0.3, modes, w, 0.3, 200.0, pos, 0.3, g)
    assert rel_l2(out, want_out) < TOL
    assert rel_l2(dv, dv_ref) < TOL, rel_l2(dv, dv_ref)
    assert rel_l2(dm, dm_ref) < TOL, rel_l2(dm, dm_ref)


def test_checkpoint_spacing_and_batching_agree():
    pot, modes, w, pos, g = _case(64, 9, 1, 5, seed=3)
    _, dv1, dm1 = _gpu_vjp(pot, modes, w, pos, g, ckpt=1)
    _, dv9, dm9 = _gpu_vjp(pot, modes, w, pos, g, ckpt=9, batch=2)
    assert rel_l2(dv9, dv1) < 1e-5
    assert rel_l2(dm9, dm1) < 1e-5
    _, dva, _ = _gpu_vjp(pot, modes, w, pos, g, ckpt=3, batch=0)
    _, dvb, _ = _gpu_vjp(pot, modes, w, pos, g, ckpt=3, batch=0)
    assert np.array_equal(dva, dvb)  # deterministic reductions


def test_autograd_through_public_stem_4d(golden):
    g = golden
    dev = torch.device("cuda")
    pot = torch.tensor(g["pot"], dtype=torch.float32, device=dev, requires_grad=True)
    mic = pb.create_microscope_config(100.0, 20.0, probe_shape=(32, 32))
    det = pb.create_detector_config(0.2, 20.0, scan_positions_px=g["positions_px"])
    beam = pb.create_probe_modes(pb.make_probe(mic, det).cpu().numpy()[..., None], [1.0], 0.2)
    slices = pb.PotentialSlices(pot, 2.0, 0.2)
    s4 = pb.stem_4d(slices, beam, mic, det)
    assert rel_l2(s4.data.detach().cpu().numpy(), g["stem4d"]) < TOL
    weights = torch.linspace(0.5, 1.5, 32 * 32, device=dev).reshape(32, 32)
    loss = (s4.data * weights).sum()
    loss.backward()
    probe = R.make_probe(100.0, 20.0, (32, 32), 20.0)
    gw = np.broadcast_to(weights.cpu().numpy(), (4, 32, 32))
    dv_ref, _ = R.stem_4d_vjp(g["pot"], 2.0, 0.2, probe[..., None], [1.0], 0.2, 100.0, g["positions_px"], 0.2, gw)
    assert rel_l2(pot.grad.cpu().numpy(), dv_ref) < TOL


def test_sum_gradient_is_null_like_reference(golden):
    """grad of sum(patterns) w.r.t. V vanishes (reference grad_pot ~1e-18)."""
    g = golden
    probe = R.make_probe(100.0, 20.0, (32, 32), 20.0)
    _, dv, _ = _gpu_vjp(g["pot"], probe[..., None], np.array([1.0]), g["positions_px"], np.ones((4, 32, 32)),
                        dz=2.0, kv=100.0, calib=0.2)
    scale = R.interaction_sigma(100.0) * 4 * 37  # sigma x total intensity
    assert np.max(np.abs(dv)) < 1e-5 * scale


def test_aberration_gradients_match_oracle_fd():
    """dL/d(defocus, C3, A1x) through make_probe_differentiable + stem_4d vs central FD in float64."""
    n, s = 64, 4
    rng = np.random.default_rng(11)
    pot = rng.uniform(0.0, 50.0, (n, n, s))
    pos = rng.uniform(-2, 2, (3, 2))
    g = rng.normal(size=(3, n, n))
    dev = torch.device("cuda")
    c1 = torch.tensor(-30.0, dtype=torch.float64, device=dev, requires_grad=True)
    c3 = torch.tensor(2e-3, dtype=torch.float64, device=dev, requires_grad=True)
    a1x = torch.tensor(5.0, dtype=torch.float64, device=dev, requires_grad=True)
    probe = pb.make_probe_differentiable(200.0, 25.0, (n, n), 30.0, c1, c3, 0.0, a1x, 0.0)
    pat = pb.stem_4d_patterns(torch.as_tensor(pot, dtype=torch.float32, device=dev), probe[..., None].contiguous(),
                              torch.ones(1, device=dev), torch.as_tensor(pos, device=dev), 1.7, 200.0, 0.3)
    loss = (pat * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum()
    loss.backward()

    def oracle_loss(d1, d3, ax):
        lam = R.relativistic_wavelength_ang(200.0)
        q = R.probe_fourier_radius((n, n), 30.0)
        f = np.fft.fftfreq(n, d=1.0 / n) / (n * 0.3)
        ly, lx = np.meshgrid(f, f, indexing="ij")
        phi = np.arctan2(ly, lx)
        chi = R.aberration(q, lam, d1, d3) + 2 * np.pi / lam * (lam * q) ** 2 / 2 * ax * np.cos(2 * phi)
        a = (q <= 0.025 / lam) * np.exp(-1j * chi)
        pr = np.fft.ifftshift(np.fft.ifft2(a))
        d = R.stem_4d(pot, 1.7, 0.3, pr[..., None], [1.0], 0.3, 200.0, pos, 0.3)["data"]
        return float(np.sum(g * d))

    for got, (args_p, args_m, h) in ((c1.grad, ((-29.9, 2e-3, 5.0), (-30.1, 2e-3, 5.0), 0.2)),
                                     (c3.grad, ((-30.0, 2.01e-3, 5.0), (-30.0, 1.99e-3, 5.0), 2e-5)),
                                     (a1x.grad, ((-30.0, 2e-3, 5.1), (-30.0, 2e-3, 4.9), 0.2))):
        fd = (oracle_loss(*args_p) - oracle_loss(*args_m)) / h
        assert abs(float(got) - fd) <= 2e-3 * max(1.0, abs(fd)), (float(got), fd)


def test_windowed_forward_and_vjp_match_oracle():
    """probe p reads the 64^2 window at windows[p] of a periodic 128^2 field (one window wraps)."""
    rng = np.random.default_rng(7)
    n, f, s = 64, 128, 3
    field = rng.uniform(0.0, 50.0, (f, f, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    windows = np.array([[0, 0], [8, 40], [64, 64], [100, 90]], np.int32)
    pos = rng.uniform(-1, 1, (4, 2))
    g = rng.normal(size=(4, n, n))
    dev = torch.device("cuda")
    out, dv, dm = pb.vjp(torch.as_tensor(field, dtype=torch.float32, device=dev),
                         torch.as_tensor(probe[..., None].astype(np.complex64), device=dev),
                         torch.ones(1, device=dev), torch.as_tensor(pos, device=dev),
                         torch.as_tensor(g, dtype=torch.float32, device=dev), 1.7, 200.0, 0.3,
                         windows=torch.as_tensor(windows, device=dev), batch=3)
    torch.cuda.synchronize()
    want = R.stem_4d_windowed(field, 1.7, 0.3, probe[..., None], [1.0], 0.3, 200.0, pos, 0.3, windows)
    dv_ref, dm_ref = R.stem_4d_windowed_vjp(field, 1.7, 0.3, probe[..., None], [1.0], 0.3, 200.0, pos, 0.3,
                                            windows, g)
    assert rel_l2(out.cpu().numpy(), want) < TOL
    assert rel_l2(dv.cpu().numpy(), dv_ref) < TOL
    assert rel_l2(dm.cpu().numpy(), dm_ref) < TOL
    # the public API agrees with the device-level call
    slices = pb.create_potential_slices(field, 1.7, 0.3)
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(n, n))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    beam = pb.create_probe_modes(probe[..., None], [1.0], 0.3)
    s4 = pb.stem_4d_windowed(slices, beam, mic, det, windows)
    assert rel_l2(s4.data.cpu().numpy(), want) < TOL


@pytest.mark.parametrize("n", [128, 256])
def test_gradient_identical_across_launch_variants(n):
    """Checkpointing forward passes in the paired kernel (at 256 also with TMA column
    blocks, tune bit 2048, and paired first / last slice passes, bit 4096) give the
    scalar kernel's residuals, hence identical gradients."""
    pot, modes, w, pos, g = _case(n, 6, 2, 4, seed=9)
    dev = torch.device("cuda")
    args = [torch.as_tensor(pot, dtype=torch.float32, device=dev), torch.as_tensor(modes.astype(np.complex64), device=dev),
            torch.as_tensor(w, dtype=torch.float32, device=dev), torch.as_tensor(pos, dtype=torch.float64, device=dev),
            torch.as_tensor(g, dtype=torch.float32, device=dev), 1.7, 200.0, 0.3]
    ref = pb.vjp(*args, ckpt_every=2, tune=3)
    for tune in (19, 147, 211, 2259, 6355, 22739):
        got = pb.vjp(*args, ckpt_every=2, tune=tune)
        for a, b in zip(ref, got):
            assert torch.equal(a, b), tune


@pytest.mark.parametrize("n,s,m,p", [(64, 4, 2, 5), (128, 3, 1, 3), (256, 2, 1, 2)])
def test_position_gradient_matches_oracle(n, s, m, p):
    pot, modes, w, pos, g = _case(n, s, m, p, seed=n)
    dev = torch.device("cuda")
    sl = torch.as_tensor(pot, dtype=torch.float32, device=dev)
    md = torch.as_tensor(modes.astype(np.complex64), device=dev)
    wt = torch.as_tensor(w, dtype=torch.float32, device=dev)
    ps = torch.as_tensor(pos, dtype=torch.float64, device=dev).requires_grad_(True)
    pat = pb.stem_4d_patterns(sl, md, wt, ps, 1.7, 200.0, 0.3)
    (pat * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()
    _, _, dpos = R.stem_4d_vjp(pot, 1.7, 0.3, modes, w, 0.3, 200.0, pos, 0.3, g, with_positions=True)
    assert rel_l2(ps.grad.cpu().numpy(), dpos) < TOL, rel_l2(ps.grad.cpu().numpy(), dpos)


@pytest.mark.parametrize("n,s,m,p", [(16, 3, 1, 3), (32, 1, 1, 2), (64, 5, 2, 3), (128, 4, 1, 5), (256, 6, 1, 3)])
def test_lambda_only_adjoint_is_bit_identical_to_lockstep(n, s, m, p):
    """With a checkpoint at every slice point the adjoint pass carries only lambda,
    two lines per thread (ms_bwd_lam.cuh); the lockstep adjoint (tune bit 65536) runs
    psi alongside and replaces it by the checkpoint at every slice point, so both give
    the same gradients bit for bit, and both match the oracle."""
    pot, modes, w, pos, g = _case(n, s, m, p, seed=n + s)
    dev = torch.device("cuda")
    args = [torch.as_tensor(pot, dtype=torch.float32, device=dev), torch.as_tensor(modes.astype(np.complex64), device=dev),
            torch.as_tensor(w, dtype=torch.float32, device=dev), torch.as_tensor(pos, dtype=torch.float64, device=dev),
            torch.as_tensor(g, dtype=torch.float32, device=dev), 1.7, 200.0, 0.3]
    base = pb.simulations.default_tune(n)
    lam = pb.vjp(*args, ckpt_every=1, tune=base, batch=2)
    lock = pb.vjp(*args, ckpt_every=1, tune=base | 65536, batch=2)
    for a, b in zip(lam, lock):
        assert torch.equal(a, b)
    dv_ref, dm_ref = R.stem_4d_vjp(pot, 1.7, 0.3, modes, w, 0.3, 200.0, pos, 0.3, g)
    assert rel_l2(lam[1].cpu().numpy(), dv_ref) < TOL
    assert rel_l2(lam[2].cpu().numpy(), dm_ref) < TOL


def test_lambda_only_adjoint_windowed_field():
    """The lambda-only adjoint on 64^2 windows of a periodic 128^2 field (one window
    wraps) equals the lockstep adjoint bit for bit."""
    rng = np.random.default_rng(17)
    n, f, s = 64, 128, 4
    dev = torch.device("cuda")
    field = torch.as_tensor(rng.uniform(0.0, 50.0, (f, f, s)), dtype=torch.float32, device=dev)
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    windows = torch.as_tensor(np.array([[0, 0], [8, 40], [64, 64], [100, 90], [120, 3]], np.int32), device=dev)
    args = [field, torch.as_tensor(probe[..., None].astype(np.complex64), device=dev), torch.ones(1, device=dev),
            torch.as_tensor(rng.uniform(-1, 1, (5, 2)), device=dev),
            torch.as_tensor(rng.normal(size=(5, n, n)), dtype=torch.float32, device=dev), 1.7, 200.0, 0.3]
    lam = pb.vjp(*args, ckpt_every=1, windows=windows, batch=3)
    lock = pb.vjp(*args, ckpt_every=1, windows=windows, batch=3, tune=pb.simulations.default_tune(n) | 65536)
    for a, b in zip(lam, lock):
        assert torch.equal(a, b)


def test_mode_weight_gradient_and_tangent_match_oracle():
    """dL/dw_m = sum_p sum_k g_p(k) I_pm(k) with I_pm the pattern of mode m alone
    (ptyro_ms_weight_grad over the stored amplitudes), and the weights' forward-mode
    tangent sum_m t_m I_pm; the oracle's per-mode patterns give both."""
    pot, modes, w, pos, g = _case(64, 4, 2, 3, seed=21)
    dev = torch.device("cuda")
    sl = torch.as_tensor(pot, dtype=torch.float32, device=dev)
    md = torch.as_tensor(modes.astype(np.complex64), device=dev)
    ps = torch.as_tensor(pos, dtype=torch.float64, device=dev)
    wt = torch.as_tensor(w, dtype=torch.float32, device=dev).requires_grad_(True)
    per_mode = [R.stem_4d(pot, 1.7, 0.3, modes[..., m:m + 1], [1.0], 0.3, 200.0, pos, 0.3)["data"] for m in range(2)]
    pat = pb.stem_4d_patterns(sl, md, wt, ps, 1.7, 200.0, 0.3)
    (pat * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()
    want = np.array([np.sum(g * per_mode[m]) for m in range(2)])
    assert rel_l2(wt.grad.cpu().numpy(), want) < TOL
    t = torch.tensor([0.3, -0.5], dtype=torch.float32, device=dev)
    _, tan = torch.func.jvp(lambda w_: pb.stem_4d_patterns(sl, md, w_, ps, 1.7, 200.0, 0.3), (wt.detach(),), (t,))
    assert rel_l2(tan.cpu().numpy(), 0.3 * per_mode[0] - 0.5 * per_mode[1]) < TOL
    # through the public stem_4d with a ProbeModes whose weights require grad
    beam = pb.ProbeModes(md, wt.detach().clone().requires_grad_(True), 0.3)
    slices = pb.create_potential_slices(sl, 1.7, 0.3)
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(64, 64))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    out = pb.stem_4d(slices, beam, mic, det)
    (out.data * torch.as_tensor(g, dtype=torch.float32, device=dev)).sum().backward()
    assert rel_l2(beam.weights.grad.cpu().numpy(), want) < TOL


@pytest.mark.parametrize("windowed", [False, True])
def test_adjoint_lanes_agree_with_one_call(windowed):
    """run_forward_ckpt and run_backward over two and three concurrent probe lanes (each its own residual
    range and side stream, dL/dV and dL/dmodes added in lane order) against one call,
    with scan-position gradients; the lanes' sums differ only by float32 rounding."""
    import ctypes
    from ptyrodactyl_b200 import _lib
    from ptyrodactyl_b200.autodiff import run_backward
    from ptyrodactyl_b200.simulations import default_tune, ms_params
    rng = np.random.default_rng(31 + windowed)
    n, S, P, M = 64, 3, 37, 2
    F = 128 if windowed else n
    dev = torch.device("cuda")
    pot = torch.as_tensor(rng.uniform(0.0, 30.0, (F, F, S)), dtype=torch.float32, device=dev)
    probe = R.make_probe(200.0, 25.0, (n, n), 25.0, defocus_ang=-30.0)
    modes = torch.as_tensor(np.stack([probe, np.roll(probe, 3, axis=0) * (0.5 + 0.2j)], -1).astype(np.complex64),
                            device=dev)
    wts = torch.tensor([0.7, 0.3], dtype=torch.float32, device=dev)
    pos = torch.as_tensor(rng.uniform(-2, 2, (P, 2)), dtype=torch.float64, device=dev)
    win = torch.as_tensor(rng.integers(0, F, (P, 2)), dtype=torch.int32, device=dev) if windowed else None
    lib = _lib.load()
    k = 1
    from ptyrodactyl_b200.simulations import check_windows
    _, f = check_windows(pot, modes, win, P)
    prm = ms_params(n, S, M, P, 200.0, 1.7, 0.25, 0.25, pot.stride(), modes.stride(), 0, default_tune(n), f, win)
    ws_b = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = torch.empty(ws_b, dtype=torch.uint8, device=dev)
    res = torch.empty(lib.ptyro_ms_residual_bytes(ctypes.byref(prm), k) // 4, dtype=torch.float32, device=dev)
    out = torch.empty((P, n, n), dtype=torch.float32, device=dev)
    _lib.check(lib.ptyro_ms_forward_ckpt(ctypes.byref(prm), k, pot.data_ptr(), modes.data_ptr(), wts.data_ptr(),
                                         pos.data_ptr(), out.data_ptr(), res.data_ptr(), ws.data_ptr(), ws_b,
                                         torch.cuda.current_stream().cuda_stream))
    # the recording forward over lanes writes the same patterns and residuals
    from ptyrodactyl_b200.autodiff import run_forward_ckpt
    for lanes in (2, 3):
        out_l, res_l = torch.empty_like(out), torch.empty_like(res)
        run_forward_ckpt(pot, modes, wts, pos, k, 1.7, 200.0, 0.25, 0.25, 0, default_tune(n), win, out_l, res_l,
                         lanes=lanes)
        assert torch.equal(out_l, out) and torch.equal(res_l, res)
    g = torch.as_tensor(rng.normal(size=(P, n, n)), dtype=torch.float32, device=dev)
    results = []
    for lanes in (1, 2, 3):
        gs, gm = torch.empty_like(pot), torch.empty_like(modes)
        gp = torch.zeros((P, 2), dtype=torch.float64, device=dev)
        run_backward(pot, modes, wts, pos, res, g, k, 1.7, 200.0, 0.25, 0.25, 0, default_tune(n), win, gs, gm, gp,
                     lanes=lanes)
        results.append((gs, gm, gp))
    for gs, gm, gp in results[1:]:
        assert torch.linalg.norm(gs - results[0][0]) <= 1e-6 * torch.linalg.norm(results[0][0])
        assert torch.linalg.norm(gm - results[0][1]) <= 1e-6 * torch.linalg.norm(results[0][1])
        assert torch.equal(gp, results[0][2])  # per-probe: the same kernels on the same probes
