"""The reference's gradient-based reconstruction loops over this engine's forward
and adjoint kernels (src/ptyrodactyl/multislice/multislice_recon.py).

Same signatures and results as ``single_slice_ptychography`` (:243-668),
``single_slice_poscorrected`` (:671-1221), ``single_slice_multi_modal``
(:1224-1737) and ``multi_slice_multi_modal`` (:1740-2227): every iteration evaluates
``stem_4d`` on the current potential, beam and (where refined) scan positions,
reduces against the measured patterns with ``_reduce_loss`` (:127-147) and applies
one optimizer step per parameter. The derivatives come from ``Stem4dFunction``'s
backward (the adjoint kernel, position gradients included).

Gradient convention: the reference steps with ``conj`` of JAX's gradient
(``_apply_optimizer_step`` :150-167), i.e. dL/dRe + i dL/dIm, which is what torch's
``.grad`` already holds; it is used unchanged.

The optimizers restate optax 0.2.3 (a dependency of the reference, absent here):
``adam`` (b1 0.9, b2 0.999, eps 1e-8, bias-corrected moments, second moment of
|g|^2 for complex parameters), ``adagrad`` (initial accumulator 0, eps 1e-8 inside
the root, zero step where the accumulator is zero) and ``rmsprop`` (decay 0.9,
eps 1e-8 inside the root, initial scale 0), with the reference's settings
(:67-86).
"""

from __future__ import annotations

from enum import Enum
from typing import Tuple, Union

import torch

from .recon import reduce_loss
from .simulations import fft2, stem_4d
from .types import (
    STEM4D,
    CalibratedArray,
    MicroscopeConfig,
    PotentialSlices,
    ProbeModes,
    create_calibrated_array,
    create_detector_config,
    create_microscope_config,
)


class LossType(str, Enum):
    """types/custom_types.py:50-67."""

    MAE = "mae"
    MSE = "mse"
    RMSE = "rmse"


def _abs_sq(g: torch.Tensor) -> torch.Tensor:
    return (g.conj() * g).real if g.is_complex() else g * g


class _Adam:
    def __init__(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps

    def init(self, p: torch.Tensor):
        return {"mu": torch.zeros_like(p), "nu": torch.zeros(p.shape, dtype=p.real.dtype, device=p.device),
                "count": 0}

    def update(self, g: torch.Tensor, st):
        mu = self.b1 * st["mu"] + (1 - self.b1) * g
        nu = self.b2 * st["nu"] + (1 - self.b2) * _abs_sq(g)
        count = st["count"] + 1
        mu_hat = mu / (1 - self.b1 ** count)
        nu_hat = nu / (1 - self.b2 ** count)
        step = -self.lr * (mu_hat / (torch.sqrt(nu_hat) + self.eps))
        return step, {"mu": mu, "nu": nu, "count": count}


class _Adagrad:
    def __init__(self, lr: float, initial_accumulator_value: float = 0.0, eps: float = 1e-8):
        self.lr, self.init_acc, self.eps = lr, initial_accumulator_value, eps

    def init(self, p: torch.Tensor):
        return {"sum": torch.full(p.shape, self.init_acc, dtype=p.real.dtype, device=p.device)}

    def update(self, g: torch.Tensor, st):
        acc = _abs_sq(g) + st["sum"]
        inv = torch.where(acc > 0, torch.rsqrt(acc + self.eps), torch.zeros_like(acc))
        return -self.lr * (inv * g), {"sum": acc}


class _RMSProp:
    def __init__(self, lr: float, decay: float = 0.9, eps: float = 1e-8, initial_scale: float = 0.0):
        self.lr, self.decay, self.eps, self.initial_scale = lr, decay, eps, initial_scale

    def init(self, p: torch.Tensor):
        return {"nu": torch.full(p.shape, self.initial_scale, dtype=p.real.dtype, device=p.device)}

    def update(self, g: torch.Tensor, st):
        nu = (1 - self.decay) * _abs_sq(g) + self.decay * st["nu"]
        return -self.lr * (g * torch.rsqrt(nu + self.eps)), {"nu": nu}


OPTIMIZERS = {
    "adam": lambda learning_rate: _Adam(float(learning_rate)),
    "adagrad": lambda learning_rate: _Adagrad(float(learning_rate), initial_accumulator_value=0.0, eps=1e-8),
    "rmsprop": lambda learning_rate: _RMSProp(float(learning_rate), decay=0.9, eps=1e-8, initial_scale=0.0),
}


def _get_optimizer(optimizer_name: str, learning_rate: float):
    if optimizer_name not in OPTIMIZERS:
        raise ValueError(f"Unknown optimizer: {optimizer_name}")
    return OPTIMIZERS[optimizer_name](learning_rate)


def _reduce(model: torch.Tensor, data: torch.Tensor, loss_mode: LossType) -> torch.Tensor:
    return reduce_loss(model, data, loss_mode.value)


def _promote(x, device) -> torch.Tensor:
    """_promote_to_complex (:208-221), as complex64 on the device."""
    t = torch.as_tensor(x.data_array if isinstance(x, CalibratedArray) else x, device=device)
    return t.to(torch.complex64).clone()


def _split_rates(learning_rate) -> Tuple[float, float]:
    lr = torch.as_tensor(learning_rate, dtype=torch.float64)
    if lr.ndim == 0:
        return float(lr), float(lr)
    return float(lr[0]), float(lr[1])


def _snapshot(buf: torch.Tensor, index: int, value: torch.Tensor) -> None:
    if 0 <= index < buf.shape[-1]:  # out-of-range snapshot indices are dropped, as in the reference
        buf[..., index] = value


class _Loop:
    """The common iteration: loss and gradients, optimizer steps, snapshots at
    iteration 0 and every ``save_every`` iterations (multislice_recon.py :575-655)."""

    def __init__(self, experimental_data: STEM4D, slice_thickness: float, loss_type: str):
        self.data = experimental_data.data
        if not self.data.is_cuda:
            self.data = self.data.to("cuda")
        self.dev = self.data.device
        self.calib = float(experimental_data.real_space_calib)
        self.dz = float(slice_thickness)
        self.positions = torch.as_tensor(experimental_data.scan_positions, dtype=torch.float64, device=self.dev)
        self.microscope: MicroscopeConfig = create_microscope_config(experimental_data.voltage_kv, 1.0)
        self.loss_mode = LossType(loss_type)

    def forward(self, pot: torch.Tensor, beam_modes: torch.Tensor, weights, positions: torch.Tensor) -> torch.Tensor:
        pots = PotentialSlices(pot.real[..., None], self.dz, self.calib)
        probe = ProbeModes(beam_modes, weights, self.calib)
        det = create_detector_config(self.calib, scan_positions_px=positions)
        return stem_4d(pots, probe, self.microscope, det).data

    def loss_and_grads(self, pot, beam_modes, weights, positions, refine_positions: bool):
        pot = pot.detach().requires_grad_(True)
        beam_modes = beam_modes.detach().requires_grad_(True)
        pos = positions.detach().requires_grad_(refine_positions)
        loss = _reduce(self.forward(pot, beam_modes, weights, pos), self.data, self.loss_mode)
        loss.backward()
        return loss.detach(), pot.grad, beam_modes.grad, (pos.grad if refine_positions else None)


def single_slice_ptychography(experimental_data: STEM4D, initial_potential: CalibratedArray,
                              initial_beam: CalibratedArray, slice_thickness: float, save_every: int = 10,
                              num_iterations: int = 1000, learning_rate: float = 0.001, loss_type: str = "mse",
                              optimizer_name: str = "adam"):
    """multislice_recon.py:243-668: refine a single potential slice and the beam.
    Returns (potential, beam, potential snapshots (H, W, S), beam snapshots)."""
    lp = _Loop(experimental_data, slice_thickness, loss_type)
    pot = _promote(initial_potential, lp.dev)
    beam = _promote(initial_beam, lp.dev)
    if not initial_beam.real_space:
        beam = fft2(beam, inverse=True)
    opt = _get_optimizer(optimizer_name, learning_rate)
    s_pot, s_beam = opt.init(pot), opt.init(beam)
    count = num_iterations // save_every
    snap_pot = torch.zeros(pot.shape + (count,), dtype=pot.dtype, device=lp.dev)
    snap_beam = torch.zeros(beam.shape + (count,), dtype=beam.dtype, device=lp.dev)
    ones = torch.ones(1, dtype=torch.float32, device=lp.dev)
    for ii in range(num_iterations):
        _, g_pot, g_beam, _ = lp.loss_and_grads(pot, beam[..., None], ones, lp.positions, False)
        step, s_pot = opt.update(g_pot, s_pot)
        pot = pot + step
        step, s_beam = opt.update(g_beam[..., 0], s_beam)
        beam = beam + step
        if ii == 0 or ii % save_every == 0:
            _snapshot(snap_pot, ii // save_every, pot)
            _snapshot(snap_beam, ii // save_every, beam)
    return (create_calibrated_array(pot, initial_potential.calib_y, initial_potential.calib_x, True),
            create_calibrated_array(beam, initial_beam.calib_y, initial_beam.calib_x, True), snap_pot, snap_beam)


def single_slice_poscorrected(experimental_data: STEM4D, initial_potential: CalibratedArray,
                              initial_beam: CalibratedArray, slice_thickness: float, save_every: int = 10,
                              num_iterations: int = 1000, learning_rate: Union[float, tuple] = 0.01,
                              loss_type: str = "mse", optimizer_name: str = "adam"):
    """multislice_recon.py:671-1221: potential, beam and scan positions; a pair of
    learning rates sets (parameters, positions). Returns (potential, beam,
    positions, potential snapshots, beam snapshots, position snapshots (P, 2, S))."""
    lp = _Loop(experimental_data, slice_thickness, loss_type)
    lr_par, lr_pos = _split_rates(learning_rate)
    opt, opt_pos = _get_optimizer(optimizer_name, lr_par), _get_optimizer(optimizer_name, lr_pos)
    pot = _promote(initial_potential, lp.dev)
    beam = _promote(initial_beam, lp.dev)
    pos = lp.positions.clone()
    s_pot, s_beam, s_pos = opt.init(pot), opt.init(beam), opt_pos.init(pos)
    count = num_iterations // save_every
    snap_pot = torch.zeros(pot.shape + (count,), dtype=pot.dtype, device=lp.dev)
    snap_beam = torch.zeros(beam.shape + (count,), dtype=beam.dtype, device=lp.dev)
    snap_pos = torch.zeros(pos.shape + (count,), dtype=pos.dtype, device=lp.dev)
    ones = torch.ones(1, dtype=torch.float32, device=lp.dev)
    for ii in range(num_iterations):
        _, g_pot, g_beam, g_pos = lp.loss_and_grads(pot, beam[..., None], ones, pos, True)
        step, s_pot = opt.update(g_pot, s_pot)
        pot = pot + step
        step, s_beam = opt.update(g_beam[..., 0], s_beam)
        beam = beam + step
        step, s_pos = opt_pos.update(g_pos, s_pos)
        pos = pos + step
        if ii == 0 or ii % save_every == 0:
            _snapshot(snap_pot, ii // save_every, pot)
            _snapshot(snap_beam, ii // save_every, beam)
            _snapshot(snap_pos, ii // save_every, pos)
    return (create_calibrated_array(pot, initial_potential.calib_y, initial_potential.calib_x, True),
            create_calibrated_array(beam, initial_beam.calib_y, initial_beam.calib_x, True), pos, snap_pot,
            snap_beam, snap_pos)


def single_slice_multi_modal(experimental_data: STEM4D, initial_pot_slice, initial_beam: ProbeModes,
                             slice_thickness: float, save_every: int = 10, num_iterations: int = 1000,
                             learning_rate: Union[float, tuple] = 0.01, loss_type: str = "mse",
                             optimizer_name: str = "adam"):
    """multislice_recon.py:1224-1737: potential slice, the beam's modes (weights
    fixed) and positions. Returns (potential, ProbeModes, positions, potential
    snapshots, mode snapshots (H, W, M, S))."""
    lp = _Loop(experimental_data, slice_thickness, loss_type)
    lr_par, lr_pos = _split_rates(learning_rate)
    opt, opt_pos = _get_optimizer(optimizer_name, lr_par), _get_optimizer(optimizer_name, lr_pos)
    pot = _promote(initial_pot_slice, lp.dev)
    modes = _promote(initial_beam.modes, lp.dev)
    weights = torch.as_tensor(initial_beam.weights, dtype=torch.float32, device=lp.dev)
    pos = lp.positions.clone()
    s_pot, s_modes, s_pos = opt.init(pot), opt.init(modes), opt_pos.init(pos)
    count = num_iterations // save_every
    snap_pot = torch.zeros(pot.shape + (count,), dtype=pot.dtype, device=lp.dev)
    snap_modes = torch.zeros(modes.shape + (count,), dtype=modes.dtype, device=lp.dev)
    for ii in range(num_iterations):
        _, g_pot, g_modes, g_pos = lp.loss_and_grads(pot, modes, weights, pos, True)
        step, s_pot = opt.update(g_pot, s_pot)
        pot = pot + step
        step, s_modes = opt.update(g_modes, s_modes)
        modes = modes + step
        step, s_pos = opt_pos.update(g_pos, s_pos)
        pos = pos + step
        if ii == 0 or ii % save_every == 0:
            _snapshot(snap_pot, ii // save_every, pot)
            _snapshot(snap_modes, ii // save_every, modes)
    beam = ProbeModes(modes, initial_beam.weights, initial_beam.calib)
    return pot, beam, pos, snap_pot, snap_modes


def multi_slice_multi_modal(experimental_data: STEM4D, initial_pot_slice, initial_beam, slice_thickness: float,
                            save_every: int = 10, num_iterations: int = 1000, learning_rate: float = 0.001,
                            pos_learning_rate: float = 0.01, loss_type: str = "mse", optimizer_name: str = "adam"):
    """multislice_recon.py:1740-2227: potential slice, beam and positions with
    separate learning rates. Returns (potential, beam, positions, potential
    snapshots, beam snapshots)."""
    lp = _Loop(experimental_data, slice_thickness, loss_type)
    opt, opt_pos = _get_optimizer(optimizer_name, learning_rate), _get_optimizer(optimizer_name, pos_learning_rate)
    pot = _promote(initial_pot_slice, lp.dev)
    beam = _promote(initial_beam, lp.dev)
    pos = lp.positions.clone()
    s_pot, s_beam, s_pos = opt.init(pot), opt.init(beam), opt_pos.init(pos)
    count = num_iterations // save_every
    snap_pot = torch.zeros(pot.shape + (count,), dtype=pot.dtype, device=lp.dev)
    snap_beam = torch.zeros(beam.shape + (count,), dtype=beam.dtype, device=lp.dev)
    ones = torch.ones(1, dtype=torch.float32, device=lp.dev)
    for ii in range(num_iterations):
        _, g_pot, g_beam, g_pos = lp.loss_and_grads(pot, beam[..., None], ones, pos, True)
        step, s_pot = opt.update(g_pot, s_pot)
        pot = pot + step
        step, s_beam = opt.update(g_beam[..., 0], s_beam)
        beam = beam + step
        step, s_pos = opt_pos.update(g_pos, s_pos)
        pos = pos + step
        if ii == 0 or ii % save_every == 0:
            _snapshot(snap_pot, ii // save_every, pot)
            _snapshot(snap_beam, ii // save_every, beam)
    return pot, beam, pos, snap_pot, snap_beam
