"""Forward-mode (tangent) kernels: parity with the oracle's linearised multislice,
the transpose identity with the adjoint kernels, and torch.func / Gauss-Newton
through the public stem_4d."""

import dataclasses

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _case(n, s, m, p, seed=0):
    rng = np.random.default_rng(seed)
    pot = rng.uniform(0.0, 60.0, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0, c3_ang=1e-3)
    modes = probe[..., None]
    if m == 2:
        modes = np.stack([probe, np.roll(probe, 2, axis=1) * (0.7 - 0.3j)], axis=-1)
    w = np.array([1.0]) if m == 1 else np.array([0.6, 0.4])
    pos = rng.uniform(-3, 3, (p, 2))
    dv = rng.normal(size=pot.shape)
    dm = (rng.normal(size=modes.shape) + 1j * rng.normal(size=modes.shape)) * np.abs(modes).max() * 0.1
    return pot, modes, w, pos, dv, dm


def _dev(*arrays):
    dev = torch.device("cuda")
    out = []
    for a in arrays:
        if a is None:
            out.append(None)
        elif np.iscomplexobj(a):
            out.append(torch.as_tensor(a.astype(np.complex64), device=dev))
        elif a.dtype == np.float64 and a.ndim == 2 and a.shape[1] == 2:
            out.append(torch.as_tensor(a, dtype=torch.float64, device=dev))
        else:
            out.append(torch.as_tensor(a, dtype=torch.float32, device=dev))
    return out


@pytest.mark.parametrize("n,s,m,p,which", [(64, 5, 1, 3, "both"), (64, 4, 2, 2, "both"), (128, 7, 1, 2, "pot"),
                                           (32, 1, 1, 3, "beam"), (256, 3, 1, 2, "both"), (16, 2, 2, 2, "both")])
def test_jvp_matches_oracle(n, s, m, p, which):
    pot, modes, w, pos, dv, dm = _case(n, s, m, p, seed=n + s)
    dv = dv if which in ("both", "pot") else None
    dm = dm if which in ("both", "beam") else None
    sl, md, wt, ps = _dev(pot, modes, w, pos)
    tsl = None if dv is None else _dev(dv)[0]
    tmd = None if dm is None else _dev(dm)[0]
    out, tan = pb.jvp(sl, md, wt, ps, tsl, tmd, 1.7, 200.0, 0.3)
    want, dwant = R.stem_4d_jvp(pot, 1.7, 0.3, modes, w, 0.3, 200.0, pos, 0.3, dslices=dv, dbeam=dm)
    assert rel_l2(out.cpu().numpy(), want) < TOL
    assert rel_l2(tan.cpu().numpy(), dwant) < TOL, rel_l2(tan.cpu().numpy(), dwant)


def test_jvp_is_the_transpose_of_the_vjp_kernels():
    n, s, p = 128, 6, 5
    pot, modes, w, pos, dv, dm = _case(n, s, 2, p, seed=11)
    g = np.random.default_rng(2).normal(size=(p, n, n))
    sl, md, wt, ps, tsl, tmd, gg = _dev(pot, modes, w, pos, dv, dm, g)
    _, tan = pb.jvp(sl, md, wt, ps, tsl, tmd, 1.7, 200.0, 0.3, batch=2)
    _, gv, gm = pb.vjp(sl, md, wt, ps, gg, 1.7, 200.0, 0.3, batch=3)
    lhs = float((tan.double() * gg.double()).sum())
    rhs = float((gv.double() * tsl.double()).sum()) + float((gm.to(torch.complex128) * tmd.to(torch.complex128)).real.sum())
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs)


def test_windowed_jvp_is_the_transpose_of_the_windowed_vjp():
    rng = np.random.default_rng(7)
    n, f, s = 64, 128, 3
    field = rng.uniform(0.0, 50.0, (f, f, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    windows = torch.as_tensor(np.array([[0, 0], [8, 40], [64, 64], [100, 90]], np.int32), device="cuda")
    pos = rng.uniform(-1, 1, (4, 2))
    g = rng.normal(size=(4, n, n))
    dv = rng.normal(size=field.shape)
    sl, md, ps, gg, tsl = _dev(field, probe[..., None], pos, g, dv)
    wt = torch.ones(1, device="cuda")
    _, tan = pb.jvp(sl, md, wt, ps, tsl, None, 1.7, 200.0, 0.3, windows=windows, batch=3)
    _, gv, _ = pb.vjp(sl, md, wt, ps, gg, 1.7, 200.0, 0.3, windows=windows, batch=3)
    lhs = float((tan.double() * gg.double()).sum())
    rhs = float((gv.double() * tsl.double()).sum())
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs)


def _public(n=64, s=4, p=6, seed=3):
    pot, modes, w, pos, dv, dm = _case(n, s, 1, p, seed=seed)
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(n, n))
    det = pb.create_detector_config(0.3, scan_positions_px=pos)
    beam = pb.create_probe_modes(modes, w, 0.3)

    def forward_fn(v):
        return pb.stem_4d(pb.PotentialSlices(v, 1.7, 0.3), beam, mic, det).data

    return forward_fn, pot, modes, w, pos, dv


def test_torch_func_jvp_through_public_stem_4d_runs_the_tangent_kernel():
    forward_fn, pot, modes, w, pos, dv = _public()
    v0, tv = _dev(pot, dv)
    before = pb._lib.load().ptyro_launch_count()
    out, tan = torch.func.jvp(forward_fn, (v0,), (tv,))
    assert pb._lib.load().ptyro_launch_count() > before
    want, dwant = R.stem_4d_jvp(pot, 1.7, 0.3, modes, w, 0.3, 200.0, pos, 0.3, dslices=dv)
    assert rel_l2(out.cpu().numpy(), want) < TOL
    assert rel_l2(tan.cpu().numpy(), dwant) < TOL
    # dual tensors (torch.autograd.forward_ad) take the same rule
    import torch.autograd.forward_ad as fwAD
    with fwAD.dual_level():
        y = forward_fn(fwAD.make_dual(v0, tv))
        assert torch.allclose(fwAD.unpack_dual(y).tangent, tan, rtol=1e-5, atol=1e-8)


def test_jtj_operator_is_symmetric_and_gauss_newton_descends():
    forward_fn, pot, modes, w, pos, dv = _public(n=64, s=3, p=4, seed=5)
    v0, a, b = _dev(pot, dv, np.random.default_rng(9).normal(size=pot.shape))
    jtj = pb.jacobian.jtj_operator(forward_fn, v0)
    ja = pb.jacobian.jvp_operator(forward_fn, v0)(a)
    jb = pb.jacobian.jvp_operator(forward_fn, v0)(b)
    lhs = float((jtj(a).double() * b.double()).sum())
    mid = float((ja.double() * jb.double()).sum())
    rhs = float((a.double() * jtj(b).double()).sum())
    assert abs(lhs - mid) <= 1e-3 * abs(mid) and abs(rhs - mid) <= 1e-3 * abs(mid)
    # a Gauss-Newton step from a perturbed potential towards synthetic data
    data = forward_fn(v0)
    start = v0 + 0.5 * torch.as_tensor(np.random.default_rng(4).normal(size=pot.shape), dtype=torch.float32,
                                       device="cuda")
    r0 = float(torch.linalg.norm(forward_fn(start) - data))
    _, rn = pb.jacobian.gauss_newton_step(forward_fn, start, data, cg_max_iterations=10, cg_tolerance=1e-8)
    assert float(rn) < 0.5 * r0


@pytest.mark.parametrize("h,w", [(64, 64), (24, 40)])
def test_forward_mode_along_scan_positions(h, w):
    """torch.func.jvp through stem_4d along a scan-position tangent (two tangent-kernel
    runs, one per axis of the shifted beam's derivative): <dI, g> against the oracle's
    position gradient, on the engine's grid and on a rectangular any-size grid."""
    rng = np.random.default_rng(h * w)
    pot = rng.uniform(0.0, 30.0, (h, w, 3))
    probe = R.make_probe(200.0, 25.0, (h, w), 30.0, defocus_ang=-30.0)
    pos = rng.uniform(-2, 2, (5, 2))
    g = rng.normal(size=(5, h, w))
    tpos = rng.normal(size=(5, 2))
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(h, w))
    pots = pb.create_potential_slices(pot, 1.7, 0.3)
    beam = pb.create_probe_modes(probe[..., None], np.array([1.0]), 0.3)
    dev = torch.device("cuda")

    det0 = pb.create_detector_config(0.3, scan_positions_px=pos)

    def fwd(p):
        return pb.stem_4d(pots, beam, mic, dataclasses.replace(det0, scan_positions_px=p)).data

    p0 = torch.tensor(pos, dtype=torch.float64, device=dev)
    out, tan = torch.func.jvp(fwd, (p0,), (torch.tensor(tpos, dtype=torch.float64, device=dev),))
    want = R.stem_4d(pot, 1.7, 0.3, probe[..., None], [1.0], 0.3, 200.0, pos, 0.3)["data"]
    assert rel_l2(out.cpu().numpy(), want) < TOL
    _, _, dpos = R.stem_4d_vjp(pot, 1.7, 0.3, probe[..., None], [1.0], 0.3, 200.0, pos, 0.3, g,
                               with_positions=True)
    got = float(np.sum(tan.cpu().numpy() * g))
    ref = float(np.sum(dpos * tpos))
    assert abs(got - ref) <= 1e-3 * abs(ref) + 1e-4 * float(np.abs(g * want).sum()) * 1e-2, (got, ref)


def test_jvp_lanes_are_bit_identical():
    """The tangent forward over two and three concurrent probe lanes writes exactly
    the patterns and tangents of one call (every output is per probe)."""
    pot, modes, w, pos, dv, dm = _case(64, 3, 2, 23, seed=4)
    sl, md, ps, tsl, tmd = _dev(pot, modes, pos, dv, dm)
    wt = torch.as_tensor(w, dtype=torch.float32, device="cuda")
    ref = pb.jvp(sl, md, wt, ps, tsl, tmd, 1.7, 200.0, 0.3, lanes=1)
    for lanes in (2, 3):
        got = pb.jvp(sl, md, wt, ps, tsl, tmd, 1.7, 200.0, 0.3, lanes=lanes)
        assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1])
