"""Carriers and factories of the multislice path, mirroring ptyrodactyl's.

Field names, factory signatures and error messages follow
``src/ptyrodactyl/types/electron_types.py`` (carriers :103-375, factories
:529-1527). Differences, all deliberate:

* arrays are ``torch.Tensor`` (CPU or CUDA) instead of JAX arrays, and keep
  float32/complex64 (the reference's factories force float64/complex128,
  ``electron_types.py:1275, :1364, :1443``; this engine computes in float32);
* traced-value checks (``eqx.error_if``) become eager ``ValueError``s with the
  reference's messages;
* scalar fields are Python floats.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from enum import Enum
from typing import Optional, Tuple

import numpy as np
import torch

Array = torch.Tensor


def as_tensor(x, dtype: torch.dtype, device=None) -> torch.Tensor:
    """numpy / torch / sequence -> tensor of ``dtype`` (device kept unless given)."""
    if isinstance(x, torch.Tensor):
        t = x
    else:
        arr = np.asarray(x)
        if arr.dtype == np.complex128 and dtype == torch.complex64:
            arr = arr.astype(np.complex64)
        elif arr.dtype == np.float64 and dtype == torch.float32:
            arr = arr.astype(np.float32)
        t = torch.from_numpy(np.ascontiguousarray(arr))
    if t.dtype != dtype:
        if dtype.is_complex and not t.dtype.is_complex:
            t = t.to(torch.float32 if dtype == torch.complex64 else torch.float64)
        t = t.to(dtype)
    if device is not None:
        t = t.to(device)
    return t


def _scalar(value, name: str) -> float:
    if isinstance(value, torch.Tensor):
        if value.numel() != 1:
            raise ValueError(f"{name} must be a scalar")
        return float(value.detach().cpu().reshape(()).item())
    arr = np.asarray(value)
    if arr.shape != ():
        raise ValueError(f"{name} must be a scalar")
    return float(arr)


def _positive(value: float, name: str) -> float:
    if not math.isfinite(value):
        raise ValueError(f"{name} must be finite")
    if value <= 0:
        raise ValueError(f"{name} must be positive")
    return value


def _finite(value: float, name: str) -> float:
    if not math.isfinite(value):
        raise ValueError(f"{name} must be finite")
    return value


def _shape_tuple(shape, name: str) -> Optional[Tuple[int, int]]:
    if shape is None:
        return None
    vals = np.asarray(shape.detach().cpu() if isinstance(shape, torch.Tensor) else shape).reshape(-1)
    if vals.shape != (2,):
        raise ValueError(f"{name} must have two entries")
    return (int(vals[0]), int(vals[1]))


class ReductionMode(str, Enum):
    """How an ensemble axis is reduced (types/distributions.py:38-52): COHERENT sums
    weighted amplitudes before |.|^2, INCOHERENT sums weighted intensities."""

    COHERENT = "coherent"
    INCOHERENT = "incoherent"


@dataclass(frozen=True)
class Distribution:
    """Weighted samples of one ensemble axis (types/distributions.py:55-102):
    samples (N, D) float64, weights (N,) float64 summing to one."""

    samples: Array
    weights: Array
    reduction: ReductionMode = ReductionMode.INCOHERENT
    axis_id: Optional[str] = None


def create_distribution(samples, weights, reduction=ReductionMode.INCOHERENT, axis_id=None) -> Distribution:
    """types/distributions.py:105-188: validated, weights clipped at zero and
    normalised to unit sum."""
    smp = as_tensor(samples, torch.float64).cpu()
    wts = as_tensor(weights, torch.float64).cpu()
    if smp.ndim != 2:
        raise ValueError("samples must have shape (N, D)")
    if wts.ndim != 1:
        raise ValueError("weights must have shape (N,)")
    if smp.shape[0] <= 0:
        raise ValueError("samples must contain at least one row")
    if smp.shape[0] != wts.shape[0]:
        raise ValueError("samples and weights must share leading dimension")
    mode = ReductionMode(reduction)
    if not bool(torch.isfinite(smp).all()):
        raise ValueError("samples must be finite")
    if not bool(torch.isfinite(wts).all()):
        raise ValueError("weights must be finite")
    if bool((wts < 0).any()):
        raise ValueError("weights must be non-negative")
    if float(wts.detach().sum()) <= 0.0:
        raise ValueError("weights must have positive total probability")
    clipped = wts.clamp(min=0.0)
    norm = clipped / clipped.sum()  # a tensor total: the normalisation's full derivative
    return Distribution(smp, norm, mode, axis_id)


@dataclass(frozen=True)
class AxisUpdate:
    """The perturbation one ensemble sample applies (electron_types.py:227-268):
    position shift in Angstrom (dy, dx), energy change in eV, tilt (x, y) in mrad;
    samples of several axes add."""

    position_delta_ang: torch.Tensor
    energy_delta_ev: torch.Tensor
    tilt_delta_mrad: torch.Tensor


def _update_field(value, shape, name: str) -> torch.Tensor:
    t = torch.zeros(shape, dtype=torch.float64) if value is None else as_tensor(value, torch.float64).cpu()
    if tuple(shape) == () and t.numel() == 1:
        t = t.reshape(())
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}")
    if not bool(torch.isfinite(t).all()):
        raise ValueError(f"{name} must be finite")
    return t


def create_axis_update(position_delta_ang=None, energy_delta_ev=None, tilt_delta_mrad=None) -> AxisUpdate:
    """electron_types.py:417-480: missing fields are zero; shapes (2,), (), (2,); finite."""
    return AxisUpdate(_update_field(position_delta_ang, (2,), "position_delta_ang"),
                      _update_field(energy_delta_ev, (), "energy_delta_ev"),
                      _update_field(tilt_delta_mrad, (2,), "tilt_delta_mrad"))


def combine_axis_updates(updates) -> AxisUpdate:
    """electron_types.py:377-414: the field-wise sum (the zero update for none)."""
    updates = tuple(updates)
    if not updates:
        return create_axis_update()
    return create_axis_update(torch.stack([u.position_delta_ang for u in updates]).sum(0),
                              torch.stack([u.energy_delta_ev for u in updates]).sum(),
                              torch.stack([u.tilt_delta_mrad for u in updates]).sum(0))


def create_trivial_distribution(sample_dim: int = 1, reduction=ReductionMode.INCOHERENT,
                                axis_id: Optional[str] = "trivial") -> Distribution:
    """types/distributions.py:190-242: one zero sample of width ``sample_dim`` with unit
    weight."""
    dim = int(sample_dim)
    if dim <= 0:
        raise ValueError("sample_dim must be positive")
    return create_distribution(torch.zeros((1, dim), dtype=torch.float64), torch.ones(1, dtype=torch.float64),
                               reduction, axis_id)


TRIVIAL_DISTRIBUTION = create_trivial_distribution()
TRIVIAL = TRIVIAL_DISTRIBUTION


@dataclass(frozen=True)
class EnsembleAxes:
    """Optional ensemble distributions (electron_types.py:74-100): a probe-mode axis
    (sample width 1: the mode index), position jitter (width 2: dy, dx in Angstrom)
    and partial coherence (width 3: dE in eV, tilt x and y in mrad)."""

    probe_modes: Optional[Distribution] = None
    position_jitter: Optional[Distribution] = None
    coherence: Optional[Distribution] = None

    def is_empty(self) -> bool:
        return self.probe_modes is None and self.position_jitter is None and self.coherence is None


@dataclass(frozen=True)
class MicroscopeConfig:
    """Microscope voltage and probe aberrations (electron_types.py:103-144)."""

    voltage_kv: float
    aperture_mrad: float
    defocus_ang: float
    c3_ang: float
    c5_ang: float
    ensemble: EnsembleAxes = field(default_factory=EnsembleAxes)
    probe_shape: Optional[Tuple[int, int]] = None


@dataclass(frozen=True)
class DetectorConfig:
    """Detector, scan and calibration (electron_types.py:147-189)."""

    real_space_calib_ang: float
    probe_calibration_pm: float
    collection_inner_mrad: float
    collection_outer_mrad: float
    scan_positions_px: Optional[Array] = None
    scan_positions_ang: Optional[Array] = None
    scan_shape: Optional[Tuple[int, int]] = None


@dataclass(frozen=True)
class AtomicSliceData:
    """Atoms, slice z bounds and per-type kernels for the atom-backed path
    (electron_types.py:192-224)."""

    atom_coords: Array
    atom_types: Array
    slice_z_bounds: Array
    atom_potentials: Array
    atom_mask: Optional[Array] = None


@dataclass(frozen=True)
class CalibratedArray:
    """2-D array with calibrations (electron_types.py:264-292)."""

    data_array: Array
    calib_y: float
    calib_x: float
    real_space: bool


@dataclass(frozen=True)
class ProbeModes:
    """Probe modes (H, W, M) and normalised weights (electron_types.py:295-317)."""

    modes: Array
    weights: Array
    calib: float


@dataclass(frozen=True)
class PotentialSlices:
    """Potential slices (H, W, S) in volt-Angstrom (electron_types.py:320-342)."""

    slices: Array
    slice_thickness: float
    calib: float


@dataclass(frozen=True)
class STEM4D:
    """4D-STEM dataset, data (P, H, W) (electron_types.py:345-373)."""

    data: Array
    real_space_calib: float
    fourier_space_calib: float
    scan_positions: Array
    voltage_kv: float


def _validate_distribution_axis(axis: Optional[Distribution], expected_axis_id: str, expected_dim: int) -> None:
    if axis is None:
        return
    if axis.samples.ndim != 2:
        raise ValueError(f"{expected_axis_id}.samples must be 2D")
    if axis.samples.shape[1] != expected_dim:
        raise ValueError(f"{expected_axis_id}.samples must have width {expected_dim}")
    if axis.weights.ndim != 1 or tuple(axis.weights.shape) != (axis.samples.shape[0],):
        raise ValueError(f"{expected_axis_id}.weights must have shape (N,)")
    if axis.axis_id not in (None, expected_axis_id):
        raise ValueError(f"{expected_axis_id}.axis_id must be {expected_axis_id!r}")


def create_ensemble_axes(probe_modes: Optional[Distribution] = None, position_jitter: Optional[Distribution] = None,
                         coherence: Optional[Distribution] = None) -> EnsembleAxes:
    """electron_types.py:488-526."""
    _validate_distribution_axis(probe_modes, "probe_modes", 1)
    _validate_distribution_axis(position_jitter, "position_jitter", 2)
    _validate_distribution_axis(coherence, "coherence", 3)
    return EnsembleAxes(probe_modes, position_jitter, coherence)


def create_microscope_config(voltage_kv, aperture_mrad, defocus_ang=0.0, c3_ang=0.0, c5_ang=0.0,
                             ensemble: Optional[EnsembleAxes] = None,
                             probe_shape=None) -> MicroscopeConfig:
    """electron_types.py:529-612."""
    voltage = _positive(_scalar(voltage_kv, "voltage_kv"), "voltage_kv")
    aperture = _positive(_scalar(aperture_mrad, "aperture_mrad"), "aperture_mrad")
    defocus = _finite(_scalar(defocus_ang, "defocus_ang"), "defocus_ang")
    c3 = _finite(_scalar(c3_ang, "c3_ang"), "c3_ang")
    c5 = _finite(_scalar(c5_ang, "c5_ang"), "c5_ang")
    return MicroscopeConfig(voltage, aperture, defocus, c3, c5,
                            EnsembleAxes() if ensemble is None else ensemble,
                            _shape_tuple(probe_shape, "probe_shape"))


def _positions(value, name: str) -> Optional[Array]:
    if value is None:
        return None
    t = as_tensor(value, torch.float64)
    if t.ndim == 1 and t.shape[0] == 2:
        t = t.reshape(1, 2)
    if t.ndim != 2 or t.shape[1] != 2:
        raise ValueError(f"{name} must have shape (P, 2)")
    if not bool(torch.isfinite(t).all()):
        raise ValueError(f"{name} contain non-finite values")
    return t


def create_detector_config(real_space_calib_ang, probe_calibration_pm=None, collection_inner_mrad=0.0,
                           collection_outer_mrad=0.0, scan_positions_px=None, scan_positions_ang=None,
                           scan_shape=None) -> DetectorConfig:
    """electron_types.py:616-731."""
    real = _positive(_scalar(real_space_calib_ang, "real_space_calib_ang"), "real_space_calib_ang")
    probe_pm = real * 100.0 if probe_calibration_pm is None else _scalar(probe_calibration_pm,
                                                                          "probe_calibration_pm")
    _positive(probe_pm, "probe_calibration_pm")
    inner = _scalar(collection_inner_mrad, "collection_inner_mrad")
    outer = _scalar(collection_outer_mrad, "collection_outer_mrad")
    if not (math.isfinite(inner) and inner >= 0):
        raise ValueError("collection_inner_mrad must be non-negative")
    if not (math.isfinite(outer) and outer >= 0):
        raise ValueError("collection_outer_mrad must be non-negative")
    if outer < inner:
        raise ValueError("collection_outer_mrad must be >= collection_inner_mrad")
    return DetectorConfig(real, probe_pm, inner, outer,
                          _positions(scan_positions_px, "scan_positions_px"),
                          _positions(scan_positions_ang, "scan_positions_ang"),
                          _shape_tuple(scan_shape, "scan_shape"))


def create_probe_modes(modes, weights, calib) -> ProbeModes:
    """electron_types.py:1238-1324: modes (H, W, M), weights (M,) normalised to sum 1."""
    m = as_tensor(modes, torch.complex64)
    w = as_tensor(weights, torch.float64)
    c = _scalar(calib, "calib")
    if m.ndim != 3:
        raise ValueError("modes must be 3D")
    if w.ndim != 1:
        raise ValueError("weights must be 1D")
    if tuple(w.shape) != (m.shape[2],):
        raise ValueError("weights must have shape (M,)")
    if not bool(torch.isfinite(torch.view_as_real(m)).all()):
        raise ValueError("modes contain non-finite values")
    if not bool(torch.isfinite(w).all()):
        raise ValueError("weights contain non-finite values")
    if bool((w < 0).any()):
        raise ValueError("weights must be non-negative")
    total = float(w.sum())
    if total <= np.finfo(np.float64).eps:
        raise ValueError("weights must sum to a positive value")
    _positive(c, "calib")
    return ProbeModes(m, (w / total).to(torch.float32), c)


def create_potential_slices(slices, slice_thickness, calib) -> PotentialSlices:
    """electron_types.py:1328-1397: slices (H, W, S) volt-Angstrom."""
    s = as_tensor(slices, torch.float32)
    if s.ndim != 3:
        raise ValueError("slices must be 3D")
    th = _scalar(slice_thickness, "slice_thickness")
    c = _scalar(calib, "calib")
    if not bool(torch.isfinite(s).all()):
        raise ValueError("slices contain non-finite values")
    _positive(th, "slice_thickness")
    _positive(c, "calib")
    return PotentialSlices(s, th, c)


def create_atomic_slice_data(atom_coords, atom_types, slice_z_bounds, atom_potentials,
                             atom_mask=None) -> AtomicSliceData:
    """electron_types.py:735-850: coords (N, 3) x, y, z Angstrom; types (N,);
    bounds (S, 2); kernels (T, H, W) volt-Angstrom; optional mask (N,)."""
    coords = as_tensor(atom_coords, torch.float64)
    types = as_tensor(atom_types, torch.int32) if not isinstance(atom_types, torch.Tensor) else atom_types.to(
        torch.int32)
    bounds = as_tensor(slice_z_bounds, torch.float64)
    pots = as_tensor(atom_potentials, torch.float32)
    mask = None if atom_mask is None else as_tensor(atom_mask, torch.float32)
    if coords.ndim != 2 or coords.shape[1] != 3:
        raise ValueError("atom_coords must have shape (N, 3)")
    if types.ndim != 1 or types.shape[0] != coords.shape[0]:
        raise ValueError("atom_types must have shape (N,)")
    if bounds.ndim != 2 or bounds.shape[1] != 2:
        raise ValueError("slice_z_bounds must have shape (S, 2)")
    if pots.ndim != 3:
        raise ValueError("atom_potentials must have shape (T, H, W)")
    if mask is not None and tuple(mask.shape) != (coords.shape[0],):
        raise ValueError("atom_mask must have shape (N,)")
    if not bool(torch.isfinite(coords).all()):
        raise ValueError("atom_coords contain non-finite values")
    if types.numel() and bool((types < 0).any()):
        raise ValueError("atom_types must be non-negative")
    if types.numel() and int(types.max()) >= pots.shape[0]:
        raise ValueError("atom_types must index atom_potentials")
    if not bool(torch.isfinite(bounds).all()):
        raise ValueError("slice_z_bounds contain non-finite values")
    if bounds.numel() and bool((bounds[:, 1] <= bounds[:, 0]).any()):
        raise ValueError("slice_z_bounds thicknesses must be positive")
    if not bool(torch.isfinite(pots).all()):
        raise ValueError("atom_potentials contain non-finite values")
    if mask is not None and not bool(torch.isfinite(mask).all()):
        raise ValueError("atom_mask contains non-finite values")
    return AtomicSliceData(coords, types, bounds, pots, mask)


def create_calibrated_array(data_array, calib_y, calib_x, real_space) -> CalibratedArray:
    """electron_types.py:853-930."""
    d = data_array if isinstance(data_array, torch.Tensor) else torch.as_tensor(np.asarray(data_array))
    if d.ndim != 2:
        raise ValueError("data_array must be 2D")
    cy = _positive(_scalar(calib_y, "calib_y"), "calib_y")
    cx = _positive(_scalar(calib_x, "calib_x"), "calib_x")
    return CalibratedArray(d, cy, cx, bool(real_space))


def create_stem4d(data, real_space_calib, fourier_space_calib, scan_positions, voltage_kv) -> STEM4D:
    """electron_types.py:1401-1527: data (P, H, W), scan_positions (P, 2)."""
    d = data if isinstance(data, torch.Tensor) else as_tensor(data, torch.float32)
    pos = as_tensor(scan_positions, torch.float64)
    if d.ndim != 3:
        raise ValueError("data must be 3D")
    if pos.ndim != 2 or pos.shape[1] != 2 or pos.shape[0] != d.shape[0]:
        raise ValueError("scan_positions must have shape (P, 2)")
    rc = _positive(_scalar(real_space_calib, "real_space_calib"), "real_space_calib")
    fc = _positive(_scalar(fourier_space_calib, "fourier_space_calib"), "fourier_space_calib")
    v = _positive(_scalar(voltage_kv, "voltage_kv"), "voltage_kv")
    return STEM4D(d, rc, fc, pos, v)
