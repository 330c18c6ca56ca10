"""Electron form factors and projected potentials of single atoms, the per-element
primitives behind ``single_atom_potential`` and ``crystal_potential_slices``
(multislice/form_factors.py, multislice/atom_potentials.py:451-536).

Host-side float64: inputs are arrays or tensors of any shape, results float64 torch
tensors on the CPU. Coefficients come from the tables ``elements.py`` loads:

* Lobato and Van Dyck (Acta Cryst. A 70 (2014) 636-649), five (a_i, b_i) pairs:
  f(g) = sum a_i (2 + b_i g^2) / (1 + b_i g^2)^2 and the projected potential
  2 pi C_MB sum [a_i / b_i K0(2 pi r / sqrt(b_i)) + a_i pi r / b_i^1.5 K1(...)],
  C_MB = 47.87801 V A^2 (the Mott-Bethe constant);
* Kirkland (Advanced Computing in Electron Microscopy), three Lorentzian (a_i, b_i)
  and three Gaussian (c_i, d_i) pairs: f(g) = sum a_i / (g^2 + b_i) + c_i exp(-d_i g^2)
  and the projected potential 4 pi^2 a0 e_k sum a_i K0(2 pi r sqrt(b_i))
  + 2 pi^2 a0 e_k sum c_i / d_i exp(-pi^2 r^2 / d_i), with the legacy a0 = 0.5292,
  e_k = 14.4.

g = q / (2 pi) in 1/Angstrom. K0 and K1 are the polynomial approximations of
Abramowitz and Stegun 9.8.5-9.8.8 (the method the reference evaluates them with);
``bessel_kv`` takes other orders from SciPy.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from .elements import _check_atom_no, _check_parameterization, kirkland_parameters, lobato_parameters

MOTT_BETHE_VOLT_ANGSTROM_SQ = 47.87801
A_BOHR = 0.529177210903  # Angstrom, CODATA 2018
_TWO_PI = 2.0 * math.pi


@dataclass(frozen=True)
class LobatoParameters:
    """Five amplitudes a_i (Angstrom) and scales b_i (Angstrom^2) of one element."""

    amplitudes: torch.Tensor
    scales: torch.Tensor


@dataclass(frozen=True)
class KirklandParameters:
    """Three Lorentzian (a_i, b_i) and three Gaussian (c_i, d_i) pairs of one element."""

    lorentzian_amplitudes: torch.Tensor
    lorentzian_scales: torch.Tensor
    gaussian_amplitudes: torch.Tensor
    gaussian_scales: torch.Tensor


def _vec(x, n: int, name: str) -> torch.Tensor:
    t = torch.as_tensor(np.asarray(x, dtype=np.float64) if not isinstance(x, torch.Tensor) else x,
                        dtype=torch.float64)
    if tuple(t.shape) != (n,):
        raise ValueError(f"{name} must have shape ({n},)")
    if not bool(torch.isfinite(t).all()):
        raise ValueError(f"{name} must be finite")
    return t


def create_lobato_parameters(amplitudes, scales) -> LobatoParameters:
    """Validated Lobato coefficients: five finite amplitudes, five positive scales."""
    b = _vec(scales, 5, "scales")
    if bool((b <= 0).any()):
        raise ValueError("scales must be positive")
    return LobatoParameters(_vec(amplitudes, 5, "amplitudes"), b)


def create_kirkland_parameters(lorentzian_amplitudes, lorentzian_scales, gaussian_amplitudes,
                               gaussian_scales) -> KirklandParameters:
    """Validated Kirkland coefficients: three finite values each, positive scales."""
    lb, gb = _vec(lorentzian_scales, 3, "lorentzian_scales"), _vec(gaussian_scales, 3, "gaussian_scales")
    if bool((lb <= 0).any()) or bool((gb <= 0).any()):
        raise ValueError("scales must be positive")
    return KirklandParameters(_vec(lorentzian_amplitudes, 3, "lorentzian_amplitudes"), lb,
                              _vec(gaussian_amplitudes, 3, "gaussian_amplitudes"), gb)


def _lobato(atom_no) -> LobatoParameters:
    row = lobato_parameters(atom_no)
    return create_lobato_parameters(row[:5], row[5:])


def _kirkland(atom_no) -> KirklandParameters:
    row = kirkland_parameters(atom_no)
    return create_kirkland_parameters(row[[0, 2, 4]], row[[1, 3, 5]], row[[6, 8, 10]], row[[7, 9, 11]])


def _out(x) -> torch.Tensor:
    return torch.from_numpy(np.array(x, dtype=np.float64))


def _as64(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy().astype(np.float64)
    return np.asarray(x, dtype=np.float64)


def _radius(r) -> np.ndarray:
    r = _as64(r)
    if not np.all(np.isfinite(r)) or np.any(r < 0.0):
        raise ValueError("r must contain finite nonnegative radial distances")
    return np.maximum(r, 1e-10)


def _k0(x: np.ndarray) -> np.ndarray:
    """K0 by Abramowitz and Stegun 9.8.5 (x <= 2, with I0) and 9.8.6 (x > 2)."""
    from scipy.special import i0
    xs = np.minimum(x, 2.0)
    t = (xs / 2.0) ** 2
    small = -np.log(xs / 2.0) * i0(xs) + (-0.57721566 + t * (0.42278420 + t * (0.23069756 + t * (
        0.03488590 + t * (0.00262698 + t * (0.00010750 + t * 0.00000740))))))
    xl = np.maximum(x, 2.0)
    y = 2.0 / xl
    large = np.exp(-xl) / np.sqrt(xl) * (1.25331414 + y * (-0.07832358 + y * (0.02189568 + y * (
        -0.01062446 + y * (0.00587872 + y * (-0.00251540 + y * 0.00053208))))))
    return np.where(x <= 2.0, small, large)


def _k1(x: np.ndarray) -> np.ndarray:
    """K1 by Abramowitz and Stegun 9.8.7 (x <= 2, with I1) and 9.8.8 (x > 2)."""
    from scipy.special import i1
    xs = np.minimum(x, 2.0)
    t = (xs / 2.0) ** 2
    small = np.log(xs / 2.0) * i1(xs) + (1.0 + t * (0.15443144 + t * (-0.67278579 + t * (
        -0.18156897 + t * (-0.01919402 + t * (-0.00110404 + t * -0.00004686)))))) / xs
    xl = np.maximum(x, 2.0)
    y = 2.0 / xl
    large = np.exp(-xl) / np.sqrt(xl) * (1.25331414 + y * (0.23498619 + y * (-0.03655620 + y * (
        0.01504268 + y * (-0.00780353 + y * (0.00325614 + y * -0.00068245))))))
    return np.where(x <= 2.0, small, large)


def bessel_kv(v: float, x) -> torch.Tensor:
    """Modified Bessel function of the second kind K_v(x), x > 0 (atom_potentials.py:
    451-536): orders 0 and 1 by Abramowitz and Stegun 9.8.5-9.8.8, order 1/2 in closed
    form sqrt(pi / (2 x)) exp(-x), other real orders from SciPy."""
    xa = _as64(x)
    v = float(v)
    if abs(v) < 1e-10:
        out = _k0(xa)
    elif abs(v - 1.0) < 1e-10:
        out = _k1(xa)
    elif abs(v - 0.5) < 1e-10:
        out = np.sqrt(math.pi / (2.0 * xa)) * np.exp(-xa)
    else:
        from scipy.special import kv
        out = kv(v, xa)
    return _out(out)


def lobato_form_factor(params: LobatoParameters, q) -> torch.Tensor:
    """f(g) = sum a_i (2 + b_i g^2) / (1 + b_i g^2)^2, g = q / (2 pi) (form_factors.py:204-243)."""
    g2 = (_as64(q) / _TWO_PI)[..., None] ** 2
    a, b = params.amplitudes.numpy(), params.scales.numpy()
    s = g2 * b
    return _out(np.sum(a * (2.0 + s) / (1.0 + s) ** 2, axis=-1))


def kirkland_form_factor(params: KirklandParameters, q) -> torch.Tensor:
    """f(g) = sum a_i / (g^2 + b_i) + sum c_i exp(-d_i g^2) (form_factors.py:246-291)."""
    g2 = (_as64(q) / _TWO_PI)[..., None] ** 2
    lor = params.lorentzian_amplitudes.numpy() / (g2 + params.lorentzian_scales.numpy())
    gau = params.gaussian_amplitudes.numpy() * np.exp(-params.gaussian_scales.numpy() * g2)
    return _out(np.sum(lor, axis=-1) + np.sum(gau, axis=-1))


def lobato_projected_potential(params: LobatoParameters, r) -> torch.Tensor:
    """Projected potential in volt-Angstrom (form_factors.py:322-371)."""
    rr = _radius(r)[..., None]
    a, b = params.amplitudes.numpy(), params.scales.numpy()
    arg = _TWO_PI * rr / np.sqrt(b)
    terms = a / b * _k0(arg) + a * math.pi * rr / b ** 1.5 * _k1(arg)
    return _out(_TWO_PI * MOTT_BETHE_VOLT_ANGSTROM_SQ * np.sum(terms, axis=-1))


def kirkland_projected_potential(params: KirklandParameters, r) -> torch.Tensor:
    """Projected potential in volt-Angstrom (form_factors.py:374-439), the three
    Lorentzian and three Gaussian terms each added in order."""
    rr = _radius(r)[..., None]
    lt = params.lorentzian_amplitudes.numpy() * _k0(_TWO_PI * rr * np.sqrt(params.lorentzian_scales.numpy()))
    d = params.gaussian_scales.numpy()
    gt = params.gaussian_amplitudes.numpy() / d * np.exp(-(math.pi ** 2) * rr ** 2 / d)
    a0, ek = 0.5292, 14.4
    return _out(4.0 * math.pi ** 2 * a0 * ek * (lt[..., 0] + lt[..., 1] + lt[..., 2])
                            + 2.0 * math.pi ** 2 * a0 * ek * (gt[..., 0] + gt[..., 1] + gt[..., 2]))


def atomic_form_factor(atom_no, q, *, parameterization: str = "lobato") -> torch.Tensor:
    """Electron form factor of element ``atom_no`` at spatial frequencies q = 2 pi g
    (form_factors.py:442-481)."""
    _check_parameterization(parameterization)
    if parameterization == "lobato":
        return lobato_form_factor(_lobato(atom_no), q)
    return kirkland_form_factor(_kirkland(atom_no), q)


def projected_atom_potential(atom_no, r, *, parameterization: str = "lobato") -> torch.Tensor:
    """Projected potential of element ``atom_no`` at radii r (form_factors.py:484-523)."""
    _check_parameterization(parameterization)
    if parameterization == "lobato":
        return lobato_projected_potential(_lobato(atom_no), r)
    return kirkland_projected_potential(_kirkland(atom_no), r)


def lobato_bandlimited_peak(atom_no, g_max) -> torch.Tensor:
    """On-nucleus peak of the Lobato potential band-limited to |g| <= g_max
    (form_factors.py:526-590): 4 pi C_MB sum a_i b_i^-1.5 [X - X / (2 (1 + X^2)) - atan(X) / 2],
    X = g_max sqrt(b_i)."""
    gm = float(_as64(g_max))
    if not math.isfinite(gm) or gm <= 0.0:
        raise ValueError("g_max must be positive and finite")
    p = _lobato(_check_atom_no(atom_no))
    a, b = p.amplitudes.numpy(), p.scales.numpy()
    x = gm * np.sqrt(b)
    anti = x - x / (2.0 * (1.0 + x * x)) - 0.5 * np.arctan(x)
    return torch.tensor(4.0 * math.pi * MOTT_BETHE_VOLT_ANGSTROM_SQ * np.sum(a * b ** -1.5 * anti),
                        dtype=torch.float64)
