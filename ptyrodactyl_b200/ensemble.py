"""Ensemble axes of the forward model: probe modes, position jitter and partial
coherence, reduced the way the reference's cbed_image ensemble branch reduces them
(multislice/simulations.py:1163-1193, bind_cbed_axes :769-888,
multislice/reduce.py:92-201).

Per Cartesian sample of the axes the reference selects a probe mode, shifts it by
the jitter, applies the coherence sample's beam tilt (a real-space phase ramp, after
stem_4d's scan shift) at the energy-shifted voltage, runs the slice loop, sums the
COHERENT axes' weighted amplitudes and the INCOHERENT axes' weighted intensities.

Here the samples become *virtual modes* of the batched engine. The slice loop is
linear in its input wave for a fixed voltage, so every incoherent combination of
samples is one virtual mode: the coherent samples' jitter-shifted modes summed with
their weights (they must share one energy and tilt), with the combination's
product weight as the mode weight and its tilt applied by the engine after the scan
shift (``ptyro_ms_forward_tilted``). Virtual modes are grouped by energy; each group
is one engine call at its voltage, accumulating into the same patterns.

A tilt is also exactly a change of the first slice's potential: the ramp
exp(i phi(r)) multiplies the shifted wave just before the first transmission
exp(i sigma V_0(r)), so it equals the transmission of V_0 + phi / sigma
(``tilt_folded_slices``, phi wrapped to [-pi, pi) so the float32 sum keeps its
precision). The derivatives through tilted samples, and tilted samples on the
any-size grids, run that way: one call per tilt, the adjoint unchanged, and
dL/dV_0 the same for the folded slice as for V_0.
"""

from __future__ import annotations

import ctypes
import itertools
import math
from typing import List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .simulations import (
    _device,
    _stream_ptr,
    _workspace,
    check_windows,
    engine_grid,
    interaction_sigma,
    fft2,
    ms_params,
    relativistic_wavelength_ang,
    run_forward_any,
)
from .types import (
    Distribution,
    EnsembleAxes,
    ProbeModes,
    ReductionMode,
    as_tensor,
    create_distribution,
)

AXIS_PROBE_MODES = "probe_modes"
AXIS_POSITION_JITTER = "position_jitter"
AXIS_COHERENCE = "coherence"
_AXIS_DIM = {AXIS_PROBE_MODES: 1, AXIS_POSITION_JITTER: 2, AXIS_COHERENCE: 3}


# ----------------------------------------------------------------------------- producers
def _normal_gauss_hermite_rule(n_quad) -> Tuple[np.ndarray, np.ndarray]:
    """Nodes and weights of the probabilists' Gauss-Hermite rule for a standard
    normal (multislice/producers.py:250-290)."""
    q = int(n_quad)
    if q <= 0:
        raise ValueError("n_quad must be positive")
    x, w = np.polynomial.hermite.hermgauss(q)
    return np.sqrt(2.0) * x, w / np.sqrt(np.pi)


def _collapse_width(width, nodes: np.ndarray, name: str) -> np.ndarray:
    arr = np.asarray(width, dtype=np.float64)
    if arr.shape != ():
        raise ValueError(f"{name} must be a scalar")
    v = float(arr)
    if not math.isfinite(v):
        raise ValueError(f"{name} must be finite")
    if v < 0.0:
        raise ValueError(f"{name} must be non-negative")
    return v * nodes if v > 0.0 else np.zeros_like(nodes)


def coherence_to_distribution(energy_spread_ev, angular_divergence_mrad, n_quad) -> Distribution:
    """Gauss-Hermite grid over (dE, tilt x, tilt y) (producers.py:46-128)."""
    nodes, weights = _normal_gauss_hermite_rule(n_quad)
    e = _collapse_width(energy_spread_ev, nodes, "energy_spread_ev")
    t = _collapse_width(angular_divergence_mrad, nodes, "angular_divergence_mrad")
    eg, txg, tyg = np.meshgrid(e, t, t, indexing="ij")
    we, wx, wy = np.meshgrid(weights, weights, weights, indexing="ij")
    samples = np.stack((eg.reshape(-1), txg.reshape(-1), tyg.reshape(-1)), axis=1)
    return create_distribution(samples, (we * wx * wy).reshape(-1), ReductionMode.INCOHERENT, AXIS_COHERENCE)


def position_jitter_to_distribution(sigma_ang, n_quad) -> Distribution:
    """Gauss-Hermite grid over (dy, dx) in Angstrom (producers.py:131-198)."""
    nodes, weights = _normal_gauss_hermite_rule(n_quad)
    d = _collapse_width(sigma_ang, nodes, "sigma_ang")
    dy, dx = np.meshgrid(d, d, indexing="ij")
    wy, wx = np.meshgrid(weights, weights, indexing="ij")
    samples = np.stack((dy.reshape(-1), dx.reshape(-1)), axis=1)
    return create_distribution(samples, (wy * wx).reshape(-1), ReductionMode.INCOHERENT, AXIS_POSITION_JITTER)


def probe_modes_to_distribution(probe: ProbeModes) -> Distribution:
    """The incoherent mode axis with the beam's weights (simulations.py:682-711)."""
    m = probe.modes.shape[2] if probe.modes.ndim == 3 else 1
    samples = np.arange(m, dtype=np.float64)[:, None]
    # a constant copy: derivatives with respect to the beam weights flow through the
    # engine calls, which take the weights themselves
    return create_distribution(samples, as_tensor(probe.weights, torch.float64).detach().cpu(),
                               ReductionMode.INCOHERENT, AXIS_PROBE_MODES)


# ----------------------------------------------------------------------------- axes
def has_extra_ensemble_axes(ensemble: EnsembleAxes) -> bool:
    """simulations.py:714-732."""
    return ensemble.probe_modes is not None or ensemble.position_jitter is not None or ensemble.coherence is not None


def ensemble_axes_for_cbed(ensemble: EnsembleAxes, beam: ProbeModes) -> Tuple[Distribution, ...]:
    """The axes cbed_image reduces over, in order (simulations.py:735-766)."""
    axes: List[Distribution] = []
    mode_count = beam.modes.shape[2] if beam.modes.ndim == 3 else 1
    if ensemble.probe_modes is not None:
        axes.append(ensemble.probe_modes)
    elif mode_count > 1:
        axes.append(probe_modes_to_distribution(beam))
    if ensemble.position_jitter is not None:
        axes.append(ensemble.position_jitter)
    if ensemble.coherence is not None:
        axes.append(ensemble.coherence)
    if not axes:
        axes.append(probe_modes_to_distribution(beam))
    return tuple(axes)


def _axis_maps(axes, mode_count: int, column_maps: Tuple[str, ...] = ()) -> Tuple[str, ...]:
    """simulations.py:1032-1127: the column map of each axis (its axis_id unless
    ``column_maps`` names them all), sample widths, probe-mode axis first."""
    if len(column_maps) not in (0, len(axes)):
        raise ValueError("column_maps must be empty or match axes length")
    maps = []
    for i, axis in enumerate(axes):
        name = column_maps[i] if column_maps else axis.axis_id
        if name is None:
            raise ValueError("distribution axis_id is required")
        if name not in _AXIS_DIM:
            raise ValueError(f"unknown axis_id {name!r}")
        if axis.samples.shape[1] != _AXIS_DIM[name]:
            raise ValueError(f"{name!r} axis must have sample width {_AXIS_DIM[name]}")
        if name == AXIS_PROBE_MODES and i != 0:
            raise ValueError("probe_modes axis must be first")
        maps.append(name)
    if AXIS_PROBE_MODES not in maps and mode_count != 1:
        raise ValueError("multimode probes require a first probe_modes axis")
    return tuple(maps)


def bind_cbed_axes(pot_slices, probe_modes: ProbeModes, microscope, detector, axes,
                   column_maps: Tuple[str, ...] = ()):
    """The per-sample amplitude of cbed_image's ensemble branch (simulations.py:
    769-888): a function of one concatenated sample row (one row of each axis, in
    order) returning the complex (H, W) detector field of the selected mode, shifted
    by the jitter at ``detector.real_space_calib_ang``, with the coherence sample's
    tilt ramp (after the shift) and energy (voltage + dE / 1000). Each call runs the
    engine's amplitude pass once. ``apply_distributions(axes, bound)`` is the ensemble
    CBED intensity."""
    from .simulations import _amplitudes_at_origin
    axes = tuple(axes)
    modes_all = probe_modes.modes if probe_modes.modes.ndim == 3 else probe_modes.modes[..., None]
    maps = _axis_maps(axes, int(modes_all.shape[2]), tuple(column_maps))
    widths = [int(a.samples.shape[1]) for a in axes]
    expected = sum(widths)
    dev = _device(pot_slices.slices.device if pot_slices.slices.is_cuda else None)
    slices = as_tensor(pot_slices.slices, torch.float32, dev)
    if slices.ndim == 2:
        slices = slices[..., None]
    modes = as_tensor(modes_all, torch.complex64, dev).contiguous()
    calib = float(detector.real_space_calib_ang)
    pot_calib = min(float(pot_slices.calib), float(probe_modes.calib))
    kv = float(microscope.voltage_kv)
    h, w = int(modes.shape[0]), int(modes.shape[1])

    def bound(sample) -> torch.Tensor:
        row = _host(torch.as_tensor(sample)).reshape(-1)
        if row.shape[0] != expected:
            raise ValueError("sample width does not match bound axes")
        mode, delta, de, tilt, c = 0, np.zeros(2), 0.0, np.zeros(2), 0
        for name, wd in zip(maps, widths):
            part = row[c:c + wd]
            c += wd
            if name == AXIS_PROBE_MODES:
                mode = int(part[0])
            elif name == AXIS_POSITION_JITTER:
                delta = delta + part
            else:
                de, tilt = de + float(part[0]), tilt + part[1:3]
        if not 0 <= mode < modes.shape[2]:
            raise ValueError(f"probe mode index {mode} out of range")
        volt = kv + de / 1000.0
        wave = modes[:, :, mode]
        if np.any(delta != 0.0):
            wave = _jitter_shift(fft2(wave[None]), delta, calib)[0]
        if np.any(tilt != 0.0):
            k = 2.0 * np.pi / relativistic_wavelength_ang(volt)
            cy = (np.arange(h, dtype=np.float64) - (h - 1) / 2.0) * calib
            cx = (np.arange(w, dtype=np.float64) - (w - 1) / 2.0) * calib
            ramp = np.exp(1j * k * ((tilt[0] / 1000.0) * cx[None, :] + (tilt[1] / 1000.0) * cy[:, None]))
            wave = wave * torch.as_tensor(ramp.astype(np.complex64), device=dev)
        amps = _amplitudes_at_origin(slices, float(pot_slices.slice_thickness), wave[:, :, None].contiguous(), volt,
                                     pot_calib)
        return amps[:, :, 0]

    return bound


class VirtualModes:
    """Virtual modes of one energy: (H, W, K) complex64 input waves, (K,) weights,
    (K, 2, n) tilt factors of the square engine grids (or None when no sample is
    tilted or the grid is not one), (K, 2) tilts in mrad (x, y), and the voltage."""

    def __init__(self, modes: torch.Tensor, weights: torch.Tensor, tilts: Optional[torch.Tensor], voltage_kv: float,
                 angles: Optional[np.ndarray] = None):
        self.modes, self.weights, self.tilts, self.voltage_kv = modes, weights, tilts, voltage_kv
        self.angles = np.zeros((modes.shape[2], 2)) if angles is None else np.asarray(angles, dtype=np.float64)


def tilt_folded_slices(slices: torch.Tensor, tilt_mrad, voltage_kv: float, calib: float) -> torch.Tensor:
    """(H, W, S) slices whose first slice carries the beam tilt: V_0 + phi / sigma with
    phi the phase of _apply_tilt_phase_ramp (simulations.py:891-946; coordinates
    (index - (size - 1) / 2) * calib, tilt (x, y) in mrad at ``voltage_kv``) wrapped to
    [-pi, pi). Out of place, so autograd passes dL/dV_0 through unchanged."""
    h, w = int(slices.shape[0]), int(slices.shape[1])
    k = 2.0 * np.pi / relativistic_wavelength_ang(voltage_kv)
    cy = (np.arange(h, dtype=np.float64) - (h - 1) / 2.0) * float(calib)
    cx = (np.arange(w, dtype=np.float64) - (w - 1) / 2.0) * float(calib)
    phase = k * ((float(tilt_mrad[0]) / 1000.0) * cx[None, :] + (float(tilt_mrad[1]) / 1000.0) * cy[:, None])
    phase = phase - 2.0 * np.pi * np.round(phase / (2.0 * np.pi))
    dv = torch.as_tensor((phase / interaction_sigma(voltage_kv)).astype(np.float32), device=slices.device)
    return torch.cat([slices[:, :, :1] + dv[:, :, None], slices[:, :, 1:]], dim=2)


def _jitter_shift(spectra: torch.Tensor, delta, calib: float) -> torch.Tensor:
    """ifft2(fft2(mode) exp(-2 pi i (qy dy + qx dx))) of (M, n, n) spectra
    (shift_beam_fourier, simulations.py:1236-1327)."""
    qy = np.fft.fftfreq(spectra.shape[-2], d=calib)
    qx = np.fft.fftfreq(spectra.shape[-1], d=calib)
    ry = np.exp(-2j * np.pi * qy * float(delta[0]))
    rx = np.exp(-2j * np.pi * qx * float(delta[1]))
    ramp = torch.as_tensor(np.outer(ry, rx).astype(np.complex64), device=spectra.device)
    return fft2(spectra * ramp, inverse=True)


def _tilt_factors(tilt_mrad, voltage_kv: float, calib: float, n: int) -> np.ndarray:
    """(2, n) factors along y and x of _apply_tilt_phase_ramp (simulations.py:891-946)."""
    lam = relativistic_wavelength_ang(voltage_kv)
    c = (np.arange(n, dtype=np.float64) - (n - 1) / 2.0) * calib
    k = 2.0 * np.pi / lam
    ty = np.exp(1j * k * (float(tilt_mrad[1]) / 1000.0) * c)
    tx = np.exp(1j * k * (float(tilt_mrad[0]) / 1000.0) * c)
    return np.stack([ty, tx])


def virtual_modes(ensemble: EnsembleAxes, beam_modes: torch.Tensor, beam: ProbeModes, voltage_kv: float,
                  calib: float, mixed: Optional[list] = None) -> List[VirtualModes]:
    """Expand the ensemble of ``beam`` into engine calls (one per energy). An
    incoherent combination whose coherent samples differ in energy or tilt is
    appended to ``mixed`` as (weight, [(wave, weight, dE, tilt), ...]) when a list is
    given, and raises ``NotImplementedError`` otherwise."""
    axes = ensemble_axes_for_cbed(ensemble, beam)
    n = beam_modes.shape[0]
    mode_count = beam_modes.shape[2]
    maps = _axis_maps(axes, mode_count)
    coherent = [i for i, a in enumerate(axes) if a.reduction is ReductionMode.COHERENT]
    incoherent = [i for i, a in enumerate(axes) if a.reduction is ReductionMode.INCOHERENT]
    samples = [a.samples.numpy() for a in axes]
    weights = [a.weights.numpy() for a in axes]
    dev = beam_modes.device
    spectra = fft2(beam_modes.permute(2, 0, 1).contiguous())  # (M, n, n)

    def update(choice):
        mode, delta, de, tilt = 0, np.zeros(2), 0.0, np.zeros(2)
        for ax, k in choice.items():
            row = samples[ax][k]
            if maps[ax] == AXIS_PROBE_MODES:
                mode = int(row[0])
            elif maps[ax] == AXIS_POSITION_JITTER:
                delta = delta + row
            else:
                de, tilt = de + float(row[0]), tilt + row[1:3]
        if not 0 <= mode < mode_count:
            raise ValueError(f"probe mode index {mode} out of range")
        return mode, delta, de, tilt

    groups = {}  # energy -> list of (wave, weight, tilt)
    for inc in itertools.product(*[range(samples[i].shape[0]) for i in incoherent]):
        w_inc = float(np.prod([weights[i][k] for i, k in zip(incoherent, inc)])) if incoherent else 1.0
        parts = []  # the coherent samples of this incoherent combination: (wave, weight, dE, tilt)
        for coh in itertools.product(*[range(samples[i].shape[0]) for i in coherent]):
            choice = dict(zip(incoherent, inc))
            choice.update(zip(coherent, coh))
            mode, delta, de, tilt = update(choice)
            w_coh = float(np.prod([weights[i][k] for i, k in zip(coherent, coh)])) if coherent else 1.0
            if np.any(delta != 0.0):
                part = _jitter_shift(spectra[mode], delta, calib)
            else:
                part = beam_modes[:, :, mode]
            parts.append((part, w_coh, de, tuple(tilt)))
        if len({(p[2], p[3]) for p in parts}) > 1:
            # a coherent sum across energies or tilts: separate operators per sample,
            # summed as amplitudes (mixed_coherent_patterns)
            if mixed is None:
                raise NotImplementedError("coherent sums over energy or tilt samples are not supported")
            mixed.append((w_inc, parts))
            continue
        wave = None
        for part, w_coh, _, _ in parts:
            wave = part * w_coh if wave is None else wave + part * w_coh
        groups.setdefault(parts[0][2], []).append((wave, w_inc, parts[0][3]))

    out = []
    square = engine_grid(beam_modes.shape[0], beam_modes.shape[1])
    for de, members in groups.items():
        volt = voltage_kv + de / 1000.0
        modes = torch.stack([m[0] for m in members], dim=2).to(torch.complex64)
        wts = torch.tensor([m[1] for m in members], dtype=torch.float32, device=dev)
        angles = np.array([np.asarray(m[2], dtype=np.float64) for m in members]).reshape(-1, 2)
        tilted = bool(np.any(angles != 0.0))
        tilts = None
        if tilted and square:
            tf = np.stack([_tilt_factors(m[2], volt, calib, n) for m in members]).astype(np.complex64)
            tilts = torch.as_tensor(tf, device=dev).contiguous()
        out.append(VirtualModes(modes, wts, tilts, volt, angles))
    return out


def run_forward_ensemble(slices: torch.Tensor, slice_thickness: float, groups: List[VirtualModes],
                         positions: torch.Tensor, calib_ang: float, shift_calib_ang: float) -> torch.Tensor:
    """Patterns (P, n, n) float32: one engine call per energy group, accumulated."""
    lib = _lib.load()
    dev = slices.device
    num_probes = positions.shape[0]
    h, w = groups[0].modes.shape[0], groups[0].modes.shape[1]
    out = torch.zeros((num_probes, h, w), dtype=torch.float32, device=dev)
    if num_probes == 0:
        return out
    if not engine_grid(h, w):  # the any-size forward, accumulating each energy's group, one call per tilt
        for g in groups:
            for tilt in np.unique(g.angles, axis=0):
                idx = np.flatnonzero(np.all(g.angles == tilt, axis=1))
                sl = slices if not np.any(tilt != 0.0) else tilt_folded_slices(slices, tilt, g.voltage_kv, calib_ang)
                sel = torch.as_tensor(idx, device=dev)
                run_forward_any(sl, slice_thickness, g.modes.index_select(2, sel).contiguous(),
                                g.weights.index_select(0, sel).contiguous(), positions, g.voltage_kv,
                                calib_ang, shift_calib_ang, out=out, accumulate=True)
        return out
    n = h
    for g in groups:
        _, f = check_windows(slices, g.modes, None, num_probes)
        prm = ms_params(n, slices.shape[2], g.modes.shape[2], num_probes, g.voltage_kv, slice_thickness, calib_ang,
                        shift_calib_ang, slices.stride(), g.modes.stride(), 0, 0, f, None,
                        _lib.PTYRO_FLAG_ACCUMULATE)
        nbytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
        if nbytes == 0:
            _lib.check(_lib.PTYRO_ERR_INVALID)
        ws = _workspace(nbytes, dev)
        if g.tilts is None:
            rc = lib.ptyro_ms_forward(ctypes.byref(prm), slices.data_ptr(), g.modes.data_ptr(), g.weights.data_ptr(),
                                      positions.data_ptr(), out.data_ptr(), ws.data_ptr(), nbytes, _stream_ptr(dev))
        else:
            rc = lib.ptyro_ms_forward_tilted(ctypes.byref(prm), slices.data_ptr(), g.modes.data_ptr(),
                                             g.weights.data_ptr(), positions.data_ptr(), g.tilts.data_ptr(),
                                             out.data_ptr(), ws.data_ptr(), nbytes, _stream_ptr(dev))
        _lib.check(rc)
    return out


class _FourierFilter(torch.autograd.Function):
    """y = ifft2(fft2(x) H) over the first two axes of (H, W, M) complex64 CUDA modes
    with a shared (H, W) filter, on the engine's transforms. Backward (torch's complex
    convention): dx = ifft2(fft2(dy) conj(H)); dH = sum_m conj(fft2(x)) fft2(dy) / (H W)."""

    @staticmethod
    def forward(ctx, x, filt):
        xk = fft2(x.permute(2, 0, 1).contiguous())
        ctx.save_for_backward(xk, filt)
        return fft2(xk * filt, inverse=True).permute(1, 2, 0).contiguous()

    @staticmethod
    def backward(ctx, gy):
        xk, filt = ctx.saved_tensors
        gk = fft2(gy.to(torch.complex64).permute(2, 0, 1).contiguous())
        gx = fft2(gk * filt.conj(), inverse=True).permute(1, 2, 0).contiguous() if ctx.needs_input_grad[0] else None
        gf = (xk.conj() * gk).sum(dim=0) / float(xk.shape[-1] * xk.shape[-2]) if ctx.needs_input_grad[1] else None
        return gx, gf


def _coherent_jitter_filter(samples: np.ndarray, weights: torch.Tensor, h: int, w: int, calib: float,
                            dev) -> torch.Tensor:
    """sum_j w_j exp(-2 pi i (qy dy_j + qx dx_j)), q = fftfreq(., calib): the coherent
    jitter sum of shift_beam_fourier's ramps as one filter (differentiable in w)."""
    qy = np.fft.fftfreq(h, d=float(calib))
    qx = np.fft.fftfreq(w, d=float(calib))
    ramps = np.exp(-2j * np.pi * (qy[None, :, None] * samples[:, 0, None, None]
                                  + qx[None, None, :] * samples[:, 1, None, None]))
    r = torch.as_tensor(ramps.astype(np.complex64), device=dev)
    return (weights.to(device=dev, dtype=torch.float32).to(torch.complex64)[:, None, None] * r).sum(dim=0)


def _host(t: torch.Tensor) -> np.ndarray:
    """A constant tensor's values as float64 NumPy, also inside a torch.func transform
    (where operations on it would be wrapped and have no storage)."""
    while torch._C._functorch.is_functorch_wrapped_tensor(t):
        t = torch._C._functorch.get_unwrapped(t)
    with torch._C._DisableFuncTorch():
        return t.detach().cpu().numpy().astype(np.float64)


def ensemble_patterns_differentiable(slices: torch.Tensor, slice_thickness: float, beam: ProbeModes,
                                     ensemble: EnsembleAxes, modes: torch.Tensor, weights: torch.Tensor,
                                     voltage_kv: float, calib_ang: float, positions: torch.Tensor,
                                     shift_calib_ang: float) -> torch.Tensor:
    """The ensemble patterns as a reverse-mode differentiable function of the
    potential, the beam modes, the beam weights and the scan positions, for
    INCOHERENT axes of probe modes, position jitter and energy spread.

    The axes form a Cartesian product (at most one axis of each kind,
    ``ensemble_axes_for_cbed``), so the patterns are
    sum_c w_c sum_j w_j stem_4d(modes, w_modes, positions + delta_j * s, voltage + dE_c),
    with s = shift_calib_ang / calib_ang: the jitter's Fourier shift at the ensemble
    calibration composes with the scan shift into one shift of the scan position.
    Each coherence sample is one differentiable engine call over all jitter copies of
    the scan, at its energy, a tilted sample with its tilt folded into the first
    slice's potential (``tilt_folded_slices``). An explicit probe-mode axis may be
    COHERENT (its modes summed with its weights into one wave), and so may the jitter
    axis (its weighted shifts are one Fourier filter of each mode, ``_FourierFilter``);
    COHERENT coherence axes raise ``NotImplementedError``. The axes' weights are
    differentiable too (the reduction's weighted sums run in torch)."""
    axes = ensemble_axes_for_cbed(ensemble, beam)
    mode_count = modes.shape[2]
    maps = _axis_maps(axes, mode_count)
    if any(a.reduction is not ReductionMode.INCOHERENT and kind == AXIS_COHERENCE for a, kind in zip(axes, maps)):
        raise NotImplementedError("derivatives through COHERENT coherence axes are not supported")
    coherent_jitter = None
    dev = slices.device
    sel, w_modes, coherent_modes = None, weights, False
    jit, w_jit = np.zeros((1, 2)), torch.ones(1, dtype=torch.float64)
    # (dE eV, tilt x mrad, tilt y mrad) -> rows of the coherence axis
    energies: dict = {(0.0, 0.0, 0.0): None}
    w_coh = torch.ones(1, dtype=torch.float64)
    for axis, kind in zip(axes, maps):
        smp = _host(axis.samples)
        if kind == AXIS_PROBE_MODES:
            idx = smp[:, 0].astype(np.int64)
            if np.any(idx < 0) or np.any(idx >= mode_count):
                raise ValueError("probe mode index out of range")
            if ensemble.probe_modes is not None:  # an explicit axis: its own weights
                sel = torch.as_tensor(idx, device=dev)
                w_modes = axis.weights.to(device=dev, dtype=torch.float32)
                coherent_modes = axis.reduction is ReductionMode.COHERENT
            elif not np.array_equal(idx, np.arange(mode_count)):
                raise ValueError("the beam's mode axis must list every mode once")
        elif kind == AXIS_POSITION_JITTER:
            if axis.reduction is ReductionMode.COHERENT:
                coherent_jitter = (smp, axis.weights)
            else:
                jit, w_jit = smp, axis.weights
        else:
            energies, w_coh = {}, axis.weights
            for r, row in enumerate(smp):
                energies.setdefault((float(row[0]), float(row[1]), float(row[2])), []).append(r)
    use_modes = modes if sel is None else modes.index_select(2, sel)
    if coherent_modes:
        # a COHERENT mode axis: one wave, the weighted sum of the selected modes
        use_modes = (use_modes * w_modes.to(use_modes.dtype)).sum(dim=2, keepdim=True)
        w_modes = torch.ones(1, dtype=torch.float32, device=dev)
    if coherent_jitter is not None:
        # a COHERENT jitter axis: the weighted sum of the shifted waves is one Fourier
        # filter of each mode (the shifts' ramps at the ensemble calibration)
        filt = _coherent_jitter_filter(coherent_jitter[0], coherent_jitter[1], int(use_modes.shape[0]),
                                       int(use_modes.shape[1]), calib_ang, dev)
        use_modes = _FourierFilter.apply(use_modes.to(torch.complex64).contiguous(), filt)
    scale = float(shift_calib_ang) / float(calib_ang)
    offsets = torch.as_tensor(jit * scale, dtype=torch.float64, device=dev)  # (J, 2)
    J, P = offsets.shape[0], positions.shape[0]
    pos_all = (positions[None, :, :] + offsets[:, None, :]).reshape(J * P, 2)
    wj = w_jit.to(device=dev, dtype=torch.float32)
    w_coh = w_coh.to(device=dev, dtype=torch.float32)
    from .autodiff import stem_4d_patterns
    out = None
    for (de, tx, ty), rows in energies.items():
        volt = voltage_kv + de / 1000.0
        sl = slices if tx == 0.0 and ty == 0.0 else tilt_folded_slices(slices, (tx, ty), volt, calib_ang)
        pat = stem_4d_patterns(sl, use_modes, w_modes.to(torch.float32), pos_all, slice_thickness,
                               volt, calib_ang, shift_calib_ang)
        w_e = w_coh[0] if rows is None else w_coh[torch.as_tensor(rows, device=dev)].sum()
        part = w_e * torch.einsum("j,jpyx->pyx", wj, pat.reshape((J, P) + tuple(pat.shape[1:])))
        out = part if out is None else out + part
    return out


def ensemble_patterns(slices: torch.Tensor, slice_thickness: float, beam: ProbeModes, ensemble: EnsembleAxes,
                      voltage_kv: float, calib_ang: float, positions: torch.Tensor,
                      shift_calib_ang: float) -> torch.Tensor:
    """Patterns with the ensemble reduced; ``calib_ang`` = min(potential, beam)
    calibration (the jitter shift and tilt ramps use it), ``shift_calib_ang`` the
    scan shift's."""
    dev = _device(slices.device)
    modes = beam.modes if beam.modes.ndim == 3 else beam.modes[..., None]
    modes = as_tensor(modes, torch.complex64, dev).contiguous()
    mixed: list = []
    groups = virtual_modes(ensemble, modes, beam, voltage_kv, calib_ang, mixed)
    if groups:
        out = run_forward_ensemble(slices, slice_thickness, groups, positions, calib_ang, shift_calib_ang)
    else:
        out = torch.zeros((positions.shape[0],) + tuple(modes.shape[:2]), dtype=torch.float32, device=dev)
    if mixed:
        mixed_coherent_patterns(out, slices, slice_thickness, mixed, voltage_kv, positions, calib_ang,
                                shift_calib_ang)
    return out


def mixed_coherent_patterns(out: torch.Tensor, slices: torch.Tensor, slice_thickness: float, mixed: list,
                            voltage_kv: float, positions: torch.Tensor, calib_ang: float, shift_calib_ang: float,
                            chunk_bytes: int = 1 << 30) -> torch.Tensor:
    """Adds sum_i w_i |sum_c w_c A(wave_c; V + dE_c, tilt_c)|^2 to ``out`` (P, n, n):
    the incoherent combinations whose coherent samples differ in energy or tilt
    (apply_distributions, reduce.py:93-201). Every coherent sample is one amplitude
    forward (``ptyro_ms_amplitudes``, fftshifted complex64, with the sample's tilt
    after the scan shift) at its voltage; the weighted amplitudes are summed and
    squared on the device, ``chunk_bytes`` of amplitudes at a time."""
    lib = _lib.load()
    dev = slices.device
    n, w = int(out.shape[1]), int(out.shape[2])
    if not engine_grid(n, w):
        raise NotImplementedError("coherent sums over energy or tilt samples need a square grid with a "
                                  "power-of-two edge")
    num_probes = positions.shape[0]
    chunk = max(1, min(num_probes, int(chunk_bytes) // (8 * n * n)))
    for w_inc, parts in mixed:
        for c0 in range(0, num_probes, chunk):
            pos = positions[c0:c0 + chunk].contiguous()
            field = None
            for wave, w_coh, de, tilt in parts:
                volt = voltage_kv + de / 1000.0
                mode = wave[:, :, None].to(torch.complex64).contiguous()
                tilts = None
                if any(t != 0.0 for t in tilt):
                    tilts = torch.as_tensor(_tilt_factors(tilt, volt, calib_ang, n)[None].astype(np.complex64),
                                            device=dev).contiguous()
                _, f = check_windows(slices, mode, None, pos.shape[0])
                prm = ms_params(n, slices.shape[2], 1, pos.shape[0], volt, slice_thickness, calib_ang,
                                shift_calib_ang, slices.stride(), mode.stride(), 0, 0, f)
                amps = torch.empty((pos.shape[0], 1, n, n), dtype=torch.complex64, device=dev)
                nbytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
                if nbytes == 0:
                    _lib.check(_lib.PTYRO_ERR_INVALID)
                ws = _workspace(nbytes, dev)
                _lib.check(lib.ptyro_ms_amplitudes(ctypes.byref(prm), slices.data_ptr(), mode.data_ptr(),
                                                   pos.data_ptr(), None if tilts is None else tilts.data_ptr(),
                                                   amps.data_ptr(), ws.data_ptr(), nbytes, _stream_ptr(dev)))
                field = amps[:, 0] * w_coh if field is None else field + amps[:, 0] * w_coh
            out[c0:c0 + chunk] += float(w_inc) * (field.real ** 2 + field.imag ** 2)
    return out
