"""Matrix-free Jacobian operators and the Gauss-Newton / Levenberg-Marquardt steps
built on them (jacobian/operators.py:30-186, jacobian/solvers.py:63-667).

``forward_fn`` maps a parameter pytree (a tensor, or tuples / lists / dicts of
tensors) to measurements. Through this package's ``stem_4d`` the products run the
hand-written kernels: ``jvp_operator`` the tangent passes (``ptyro_ms_jvp``),
``vjp_operator`` the checkpointed forward and the adjoint passes.

Complex parameters: JAX's ``vjp`` of a real output returns ``conj(2 dL/dconj z)``
and the reference's solvers conjugate it (``_tree_conj``) to get the real-Hermitian
normal operator; torch's ``vjp`` already returns ``2 dL/dconj z``, so the steps
below match the reference's without that conjugation.
"""

from __future__ import annotations

from typing import Callable, Tuple

import torch
from torch.utils import _pytree as pytree

Tree = object


def _leaves(t: Tree):
    return pytree.tree_leaves(t)


def _map(f, *trees):
    return pytree.tree_map(f, *trees)


def tree_dot(a: Tree, b: Tree) -> torch.Tensor:
    """sum over leaves of Re(vdot(a, b)) (jacobian/_treemath.py:63-100)."""
    terms = [torch.vdot(x.reshape(-1), y.reshape(-1)).real for x, y in zip(_leaves(a), _leaves(b))]
    return torch.stack(terms).sum() if terms else torch.zeros(())


def _axpy(alpha, x: Tree, y: Tree) -> Tree:
    return _map(lambda u, v: v + alpha * u, x, y)


def jvp_operator(forward_fn: Callable[[Tree], torch.Tensor], params: Tree) -> Callable[[Tree], torch.Tensor]:
    """J v at ``params`` by forward-mode differentiation (operators.py:30-80)."""

    def jvp_fn(tangent_vector: Tree) -> torch.Tensor:
        _, out_tangent = torch.func.jvp(forward_fn, (params,), (tangent_vector,))
        return out_tangent

    return jvp_fn


def vjp_operator(forward_fn: Callable[[Tree], torch.Tensor], params: Tree) -> Callable[[torch.Tensor], Tree]:
    """J^T u at ``params`` (operators.py:83-130); the forward (with its residuals)
    runs once, every call runs the pullback."""
    _, pullback = torch.func.vjp(forward_fn, params)

    def vjp_fn(cotangent_vector: torch.Tensor) -> Tree:
        return pullback(cotangent_vector)[0]

    return vjp_fn


def jtj_operator(forward_fn: Callable[[Tree], torch.Tensor], params: Tree) -> Callable[[Tree], Tree]:
    """J^T J v: a JVP followed by the cached pullback (operators.py:133-186)."""
    _, pullback = torch.func.vjp(forward_fn, params)

    def jtj_fn(vector: Tree) -> Tree:
        _, forward_tangent = torch.func.jvp(forward_fn, (params,), (vector,))
        return pullback(forward_tangent)[0]

    return jtj_fn


def hvp_gauss_newton(forward_fn: Callable[[Tree], torch.Tensor], params: Tree,
                     residual: torch.Tensor) -> Callable[[Tree], Tree]:
    """Gauss-Newton Hessian-vector product = J^T J (operators.py:188-236);
    ``residual`` is accepted for API consistency and unused."""
    del residual
    return jtj_operator(forward_fn, params)


def conjugate_gradient(linear_operator: Callable[[Tree], Tree], rhs: Tree, x0: Tree, max_iterations: int = 100,
                       tolerance: float = 1e-6) -> Tuple[Tree, int]:
    """CG on a symmetric positive semi-definite operator (solvers.py:63-181):
    the same recurrence and 1e-12 guards; iterations stop once r.r < tol^2 (the
    reference keeps the state frozen from there on, which gives the same x)."""
    r = _map(lambda b, ax: b - ax, rhs, linear_operator(x0))
    x, p = x0, r
    rr = tree_dot(r, r)
    tol2 = tolerance ** 2
    it = 0
    for _ in range(int(max_iterations)):
        if float(rr) < tol2:
            break
        ap = linear_operator(p)
        alpha = rr / (tree_dot(p, ap) + 1e-12)
        x = _axpy(alpha, p, x)
        r = _axpy(-alpha, ap, r)
        rr_new = tree_dot(r, r)
        beta = rr_new / (rr + 1e-12)
        p = _axpy(beta, p, r)
        rr = rr_new
        it += 1
    return x, it


def gauss_newton_step(forward_fn: Callable[[Tree], torch.Tensor], params: Tree, data: torch.Tensor,
                      cg_max_iterations: int = 50, cg_tolerance: float = 1e-6) -> Tuple[Tree, torch.Tensor]:
    """One Gauss-Newton update (solvers.py:184-265): solve J^T J d = J^T r by CG,
    params - d, and the residual norm there."""
    prediction, pullback = torch.func.vjp(forward_fn, params)
    residual = prediction - data
    gradient = pullback(residual)[0]

    def jtj_fn(v: Tree) -> Tree:
        _, jv = torch.func.jvp(forward_fn, (params,), (v,))
        return pullback(jv)[0]

    x0 = _map(torch.zeros_like, params)
    step, _ = conjugate_gradient(jtj_fn, gradient, x0, cg_max_iterations, cg_tolerance)
    new_params = _map(lambda a, b: a - b, params, step)
    new_residual = forward_fn(new_params) - data
    return new_params, torch.sqrt(torch.sum(new_residual ** 2))


def levenberg_marquardt_step(forward_fn: Callable[[Tree], torch.Tensor], params: Tree, data: torch.Tensor,
                             damping, cg_max_iterations: int = 50,
                             cg_tolerance: float = 1e-6) -> Tuple[Tree, torch.Tensor, torch.Tensor]:
    """One Levenberg-Marquardt update with gain-ratio damping control
    (solvers.py:388-522): damping / 3 above a gain of 0.75, x 2 below 0.25; the
    step is kept when the gain is positive."""
    prediction, pullback = torch.func.vjp(forward_fn, params)
    residual = prediction - data
    rss = torch.sum(residual ** 2)
    gradient = pullback(residual)[0]
    damping = torch.as_tensor(damping, dtype=rss.dtype, device=rss.device)

    def jtj_fn(v: Tree) -> Tree:
        _, jv = torch.func.jvp(forward_fn, (params,), (v,))
        return pullback(jv)[0]

    def damped(v: Tree) -> Tree:
        return _axpy(damping, v, jtj_fn(v))

    x0 = _map(torch.zeros_like, params)
    step, _ = conjugate_gradient(damped, gradient, x0, cg_max_iterations, cg_tolerance)
    candidate = _map(lambda a, b: a - b, params, step)
    new_rss = torch.sum((forward_fn(candidate) - data) ** 2)
    actual = rss - new_rss
    predicted = tree_dot(step, gradient) - 0.5 * tree_dot(step, jtj_fn(step))
    gain = actual / (predicted + 1e-12)
    if float(gain) > 0.75:
        new_damping = damping / 3.0
    elif float(gain) < 0.25:
        new_damping = damping * 2.0
    else:
        new_damping = damping
    if float(gain) > 0.0:
        return candidate, torch.sqrt(new_rss), new_damping
    return params, torch.sqrt(rss), new_damping
