"""Jacobian operators and GN/LM steps on CPU through a plain torch model
(the same host logic that drives the engine's kernels on the GPU)."""

import torch

from ptyrodactyl_b200 import jacobian as J


def _model():
    g = torch.Generator().manual_seed(0)
    a = torch.randn(12, 5, generator=g, dtype=torch.float64)

    def f(p):
        return torch.tanh(a @ p["x"]) + p["y"].abs() ** 2 @ torch.ones(3, 12, dtype=torch.float64)

    params = {"x": torch.randn(5, generator=g, dtype=torch.float64),
              "y": torch.randn(3, generator=g, dtype=torch.complex128)}
    return f, params


def _flat_jacobian(f, params):
    x, y = params["x"], params["y"]

    def g(xr, yr, yi):
        return f({"x": xr, "y": torch.complex(yr, yi)})

    jx, jyr, jyi = torch.autograd.functional.jacobian(g, (x, y.real.clone(), y.imag.clone()))
    return torch.cat([jx, jyr, jyi], dim=1)


def _flat(t):
    return torch.cat([t["x"], t["y"].real, t["y"].imag])


def test_jvp_and_jtj_match_the_explicit_jacobian():
    f, params = _model()
    jm = _flat_jacobian(f, params)
    v = {"x": torch.randn(5, dtype=torch.float64), "y": torch.randn(3, dtype=torch.complex128)}
    jv = J.jvp_operator(f, params)(v)
    assert torch.allclose(jv, jm @ _flat(v), atol=1e-10)
    u = torch.randn(12, dtype=torch.float64)
    ju = J.vjp_operator(f, params)(u)
    # torch's pullback of a complex leaf is dL/dRe + i dL/dIm
    assert torch.allclose(_flat(ju), jm.T @ u, atol=1e-10)
    jtj = J.jtj_operator(f, params)(v)
    assert torch.allclose(_flat(jtj), jm.T @ (jm @ _flat(v)), atol=1e-10)
    assert torch.allclose(_flat(J.hvp_gauss_newton(f, params, None)(v)), _flat(jtj))


def test_conjugate_gradient_solves_spd_system():
    g = torch.Generator().manual_seed(3)
    m = torch.randn(8, 8, generator=g, dtype=torch.float64)
    a = m @ m.T + 8 * torch.eye(8, dtype=torch.float64)
    b = torch.randn(8, generator=g, dtype=torch.float64)
    x, it = J.conjugate_gradient(lambda v: a @ v, b, torch.zeros(8, dtype=torch.float64), 100, 1e-6)
    assert torch.allclose(a @ x, b, atol=1e-5) and 0 < it <= 12


def test_gauss_newton_solves_linear_least_squares_in_one_step():
    g = torch.Generator().manual_seed(5)
    a = torch.randn(20, 6, generator=g, dtype=torch.float64)
    y = torch.randn(20, generator=g, dtype=torch.float64)
    p, rn = J.gauss_newton_step(lambda p: a @ p, torch.zeros(6, dtype=torch.float64), y, 100, 1e-9)
    want = torch.linalg.lstsq(a, y[:, None]).solution[:, 0]
    assert torch.allclose(p, want, atol=1e-8)
    assert abs(float(rn) - float(torch.linalg.norm(a @ want - y))) < 1e-8


def test_levenberg_marquardt_damping_control():
    f, params = _model()
    data = f({"x": params["x"] * 0.5, "y": params["y"]})
    new, rn, damp = J.levenberg_marquardt_step(f, params, data, 1.0, 50, 1e-10)
    before = float(torch.linalg.norm(f(params) - data))
    assert float(rn) < before and float(damp) in (1.0 / 3.0, 1.0, 2.0)
    # a huge step that cannot reduce the residual is rejected and the damping grows
    same, rn2, damp2 = J.levenberg_marquardt_step(f, new, f(new), 1e-3, 50, 1e-10)
    assert float(rn2) <= 1e-12 or float(damp2) == 2e-3
