"""The late distribution reducers (reduce.py) on toy bound fields, the reference's
own cases (tests/test_ptyrodactyl/test_multislice/test_reduce.py): hand-computed
coherent and incoherent sums, the trivial axis, gradients through the weights and
through the bound closure, the cursor order and one-axis agreement. CPU only."""

import pytest
import torch

import ptyrodactyl_b200 as pb

C = pb.ReductionMode.COHERENT
I = pb.ReductionMode.INCOHERENT


def _t(v):
    return torch.tensor(v, dtype=torch.float64)


def _c(v):
    return torch.tensor(v, dtype=torch.complex128)


def _scalar_field(s):
    x = s[0]
    return torch.stack([torch.stack([x + 1j * (x + 1.0), 2.0 * x - 0.5j]),
                        torch.stack([x - 1.0j, -x + 0.25j])]).to(torch.complex128)


def _param_field(s, p):
    x, y = s[0], s[1]
    return torch.stack([torch.stack([p * x + 1j * (y + 1.0), x - 1j * p]),
                        torch.stack([p + 0.5j * y, x + p * y + 1.0j])]).to(torch.complex128)


def _cursor_field(c):
    a, u, v = c[0], c[1], c[2]
    return torch.stack([torch.stack([a + 1j * u, v - 1j * a]),
                        torch.stack([u * v + 0.25j, a + u + v + 0.5j])]).to(torch.complex128)


A0 = [[1.0 + 2.0j, 2.0 - 0.5j], [1.0 - 1.0j, -1.0 + 0.25j]]
A1 = [[2.0 + 3.0j, 4.0 - 0.5j], [2.0 - 1.0j, -2.0 + 0.25j]]


def test_coherent_sums_then_squares():
    d = pb.create_distribution(_t([[1.0], [2.0]]), _t([0.25, 0.75]), C)
    want = (0.25 * _c(A0) + 0.75 * _c(A1)).abs() ** 2
    assert torch.allclose(pb.apply_distribution(d, _scalar_field), want, rtol=1e-12, atol=1e-12)


def test_incoherent_squares_then_sums():
    d = pb.create_distribution(_t([[1.0], [2.0]]), _t([0.25, 0.75]), I)
    want = 0.25 * _c(A0).abs() ** 2 + 0.75 * _c(A1).abs() ** 2
    assert torch.allclose(pb.apply_distribution(d, _scalar_field), want, rtol=1e-12, atol=1e-12)


def test_trivial_axis_is_the_modulus_square():
    want = _scalar_field(pb.TRIVIAL.samples[0]).abs() ** 2
    assert torch.equal(pb.apply_distribution(pb.TRIVIAL, _scalar_field), want)
    t = pb.create_trivial_distribution(3, C, "t")
    assert t.samples.shape == (1, 3) and t.reduction is C and float(t.weights[0]) == 1.0
    with pytest.raises(ValueError, match="sample_dim must be positive"):
        pb.create_trivial_distribution(0)


@pytest.mark.parametrize("mode", [C, I])
def test_gradients_through_weights_and_bound_parameter(mode):
    samples = _t([[0.1, -0.2], [0.3, 0.4], [-0.5, 0.7]])
    w = _t([0.2, 0.3, 0.5]).requires_grad_(True)
    d = pb.create_distribution(samples, w, mode, "grad")
    pb.apply_distribution(d, lambda s: _param_field(s, torch.tensor(0.8, dtype=torch.float64))).sum().backward()
    assert w.grad.shape == (3,) and bool(torch.isfinite(w.grad).all())
    # the normalisation's full derivative: scaling all weights changes nothing
    assert abs(float((w.grad * w.detach()).sum())) < 1e-12
    p = torch.tensor(0.8, dtype=torch.float64, requires_grad=True)
    d2 = pb.create_distribution(samples, _t([0.2, 0.3, 0.5]), mode, "grad")
    pb.apply_distribution(d2, lambda s: _param_field(s, p)).sum().backward()
    assert bool(torch.isfinite(p.grad))
    # against central differences of the reducer itself
    eps = 1e-6
    hi = pb.apply_distribution(d2, lambda s: _param_field(s, torch.tensor(0.8 + eps, dtype=torch.float64))).sum()
    lo = pb.apply_distribution(d2, lambda s: _param_field(s, torch.tensor(0.8 - eps, dtype=torch.float64))).sum()
    assert abs(float(p.grad) - float(hi - lo) / (2 * eps)) < 1e-6


def test_mixed_coherent_and_incoherent_axes():
    coh = pb.create_distribution(_t([[1.0], [2.0]]), _t([0.25, 0.75]), C, "coherent")
    inc = pb.create_distribution(_t([[10.0, -1.0], [20.0, 0.5]]), _t([0.4, 0.6]), I, "incoherent")

    def f(a, u, v):
        return _cursor_field(_t([a, u, v]))
    want = (0.4 * (0.25 * f(1, 10, -1) + 0.75 * f(2, 10, -1)).abs() ** 2
            + 0.6 * (0.25 * f(1, 20, 0.5) + 0.75 * f(2, 20, 0.5)).abs() ** 2)
    assert torch.allclose(pb.apply_distributions((coh, inc), _cursor_field), want, rtol=1e-12, atol=1e-12)
    # hand-written field values of the same cursors
    assert torch.equal(f(1, 10, -1), _c([[1.0 + 10.0j, -1.0 - 1.0j], [-10.0 + 0.25j, 10.0 + 0.5j]]))
    assert torch.equal(f(2, 20, 0.5), _c([[2.0 + 20.0j, 0.5 - 2.0j], [10.0 + 0.25j, 22.5 + 0.5j]]))


def test_cursor_concatenates_rows_in_tuple_order():
    a = pb.create_distribution(_t([[2.0]]), _t([1.0]), C, "first")
    b = pb.create_distribution(_t([[3.0, 5.0]]), _t([1.0]), C, "second")

    def echo(c):
        return torch.stack([torch.stack([c[0] + 1j * c[1], c[2] + 0j]),
                            torch.stack([c[0] + 1j * c[2], c[1] + 0j])]).to(torch.complex128)
    want = _c([[2.0 + 3.0j, 5.0], [2.0 + 5.0j, 3.0]]).abs() ** 2
    assert torch.equal(pb.apply_distributions((a, b), echo), want)


@pytest.mark.parametrize("mode", [C, I])
def test_single_axis_agrees(mode):
    d = pb.create_distribution(_t([[-1.0], [0.5], [2.0]]), _t([0.2, 0.3, 0.5]), mode, "single")
    assert torch.allclose(pb.apply_distribution(d, _scalar_field), pb.apply_distributions((d,), _scalar_field),
                          rtol=1e-12, atol=1e-12)


def test_no_axes_rejected():
    with pytest.raises(ValueError, match="at least one axis"):
        pb.apply_distributions((), _scalar_field)


def test_axis_updates_add_field_by_field():
    a = pb.create_axis_update(position_delta_ang=[0.1, -0.2], energy_delta_ev=0.5)
    b = pb.create_axis_update(tilt_delta_mrad=[1.0, 2.0], energy_delta_ev=-0.25)
    c = pb.combine_axis_updates((a, b))
    assert torch.equal(c.position_delta_ang, _t([0.1, -0.2]))
    assert float(c.energy_delta_ev) == 0.25 and torch.equal(c.tilt_delta_mrad, _t([1.0, 2.0]))
    z = pb.combine_axis_updates(())
    assert float(z.energy_delta_ev) == 0.0 and not bool(z.position_delta_ang.any())
    with pytest.raises(ValueError, match="shape"):
        pb.create_axis_update(position_delta_ang=[1.0, 2.0, 3.0])
    with pytest.raises(ValueError, match="finite"):
        pb.create_axis_update(energy_delta_ev=float("nan"))
