"""Validated entry points (src/ptyrodactyl/multislice/checked.py): the same checks
and messages as the reference, then the engine.

Structural problems raise ``ValueError`` (the reference's ``_raise_if``). Value
problems, which the reference reports from inside its traced computation through
``eqx.error_if`` (an ``EquinoxRuntimeError``, a ``RuntimeError``), raise
:class:`CheckedValueError`, a ``RuntimeError`` with the reference's message.
"""

from __future__ import annotations

import math
from typing import Optional, Tuple

import torch

from .simulations import cbed_image, make_probe, stem4d_sharded, stem_4d
from .types import (
    AtomicSliceData,
    CalibratedArray,
    DetectorConfig,
    MicroscopeConfig,
    PotentialSlices,
    ProbeModes,
    STEM4D,
    create_atomic_slice_data,
)


class CheckedValueError(RuntimeError):
    """A value check failed (the reference's eqx.error_if)."""


def _raise_if(condition: bool, message: str) -> None:
    if condition:
        raise ValueError(message)


def _error_if(condition: bool, message: str) -> None:
    if condition:
        raise CheckedValueError(message)


def _shape(x) -> Tuple[int, ...]:
    return tuple(x.shape) if hasattr(x, "shape") else tuple(torch.as_tensor(x).shape)


def _all_finite(x) -> bool:
    t = torch.as_tensor(x)
    if t.is_complex():
        t = torch.view_as_real(t)
    return bool(torch.isfinite(t).all())


def _scalar(value, name: str) -> float:
    t = torch.as_tensor(value)
    _raise_if(t.ndim != 0, f"{name} must be a scalar")
    return float(t)


def _positive(value, name: str) -> None:
    v = _scalar(value, name)
    _error_if(not math.isfinite(v), f"{name} must be finite")
    _error_if(v <= 0, f"{name} must be positive")


def _finite(value, name: str) -> None:
    _error_if(not math.isfinite(_scalar(value, name)), f"{name} must be finite")


def _nonnegative(value, name: str) -> None:
    v = _scalar(value, name)
    _error_if(not math.isfinite(v), f"{name} must be finite")
    _error_if(v < 0, f"{name} must be non-negative")


def _checked_microscope(m: MicroscopeConfig) -> None:
    """checked.py _checked_microscope."""
    _positive(m.voltage_kv, "voltage_kv")
    _positive(m.aperture_mrad, "aperture_mrad")
    _finite(m.defocus_ang, "defocus_ang")
    _finite(m.c3_ang, "c3_ang")
    _finite(m.c5_ang, "c5_ang")


def _checked_detector(d: DetectorConfig) -> None:
    """checked.py _checked_detector."""
    _nonnegative(d.collection_inner_mrad, "collection_inner_mrad")
    _nonnegative(d.collection_outer_mrad, "collection_outer_mrad")
    _error_if(float(d.collection_outer_mrad) < float(d.collection_inner_mrad),
              "collection_outer_mrad must be >= collection_inner_mrad")
    _positive(d.real_space_calib_ang, "real_space_calib_ang")
    _positive(d.probe_calibration_pm, "probe_calibration_pm")
    if d.scan_positions_px is not None:
        _error_if(not _all_finite(d.scan_positions_px), "scan_positions_px contain non-finite values")
    if d.scan_positions_ang is not None:
        _error_if(not _all_finite(d.scan_positions_ang), "scan_positions_ang contain non-finite values")


def _potential_grid_shape(p: PotentialSlices, name: str) -> Tuple[int, int]:
    s = _shape(p.slices)
    _raise_if(len(s) not in (2, 3), f"{name}.slices must be 2D or 3D")
    return s[0], s[1]


def _beam_grid_shape(beam: ProbeModes, name: str) -> Tuple[int, int]:
    ms, ws = _shape(beam.modes), _shape(beam.weights)
    _raise_if(len(ms) not in (2, 3), f"{name}.modes must be 2D or 3D")
    _raise_if(len(ws) != 1, f"{name}.weights must be 1D")
    m = 1 if len(ms) == 2 else ms[2]
    _raise_if(ws != (m,), f"{name}.weights must have shape (M,)")
    return ms[0], ms[1]


def _validate_cbed_structure(p: PotentialSlices, beam: ProbeModes, pot_name: str) -> None:
    _raise_if(_beam_grid_shape(beam, "beam") != _potential_grid_shape(p, pot_name),
              f"beam.modes spatial shape must match {pot_name}.slices")


def _checked_potential_slices(p: PotentialSlices, name: str) -> None:
    _error_if(not _all_finite(p.slices), f"{name}.slices contain non-finite values")
    _error_if(not math.isfinite(float(p.slice_thickness)), f"{name}.slice_thickness must be finite")
    _error_if(float(p.slice_thickness) <= 0, f"{name}.slice_thickness must be positive")
    _error_if(not math.isfinite(float(p.calib)), f"{name}.calib must be finite")
    _error_if(float(p.calib) <= 0, f"{name}.calib must be positive")


def _checked_beam(beam: ProbeModes) -> None:
    _error_if(not _all_finite(beam.modes), "beam.modes contain non-finite values")
    _error_if(not _all_finite(beam.weights), "beam.weights contain non-finite values")
    _error_if(not math.isfinite(float(beam.calib)), "beam.calib must be finite")
    _error_if(float(beam.calib) <= 0, "beam.calib must be positive")


def _validate_positions_structure(positions, name: str) -> None:
    s = _shape(positions)
    _raise_if(len(s) != 2, f"{name} must be 2D")
    _raise_if(s[1] != 2, f"{name} must have shape (P, 2)")


def _checked_positions_in_pixels(positions, grid_shape: Tuple[int, int]) -> None:
    t = torch.as_tensor(positions, dtype=torch.float64)
    _error_if(not _all_finite(t), "positions contain non-finite values")
    h, w = grid_shape
    _error_if(bool(((t[:, 0] < 0) | (t[:, 1] < 0) | (t[:, 0] >= h) | (t[:, 1] >= w)).any()),
              "positions must be within pot_slice grid bounds")


def checked_make_probe(microscope: MicroscopeConfig, detector: DetectorConfig) -> torch.Tensor:
    """checked.py checked_make_probe."""
    _raise_if(microscope.probe_shape is None, "microscope.probe_shape is required")
    _checked_microscope(microscope)
    _checked_detector(detector)
    return make_probe(microscope, detector)


def checked_cbed_image(pot_slices: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig) -> CalibratedArray:
    """checked.py checked_cbed_image."""
    _validate_cbed_structure(pot_slices, beam, "pot_slices")
    _checked_potential_slices(pot_slices, "pot_slices")
    _checked_beam(beam)
    _checked_microscope(microscope)
    return cbed_image(pot_slices, beam, microscope)


def checked_stem_4d(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
                    detector: DetectorConfig) -> STEM4D:
    """checked.py:887: the structure, value and position-bounds checks, then stem_4d."""
    _validate_cbed_structure(pot_slice, beam, "pot_slice")
    if detector.scan_positions_px is None:
        raise ValueError("detector.scan_positions_px is required")
    _validate_positions_structure(detector.scan_positions_px, "positions")
    _checked_potential_slices(pot_slice, "pot_slice")
    _checked_beam(beam)
    _checked_positions_in_pixels(detector.scan_positions_px, _potential_grid_shape(pot_slice, "pot_slice"))
    _checked_microscope(microscope)
    _checked_detector(detector)
    return stem_4d(pot_slice, beam, microscope, detector)


def checked_stem4d_sharded(probe_modes: ProbeModes, sample: AtomicSliceData, microscope: MicroscopeConfig,
                           detector: DetectorConfig, mesh=None) -> STEM4D:
    """checked.py checked_stem4d_sharded."""
    pos = detector.scan_positions_ang
    if pos is None:
        raise ValueError("detector.scan_positions_ang is required")
    ps, ss = _shape(probe_modes.modes), _shape(pos)
    cs, ts = _shape(sample.atom_coords), _shape(sample.atom_types)
    bs, vs = _shape(sample.slice_z_bounds), _shape(sample.atom_potentials)
    _raise_if(len(ps) != 3, "probe_modes must be 3D")
    _raise_if(len(ss) != 2, "scan_positions_ang must be 2D")
    _raise_if(ss[1] != 2, "scan_positions_ang must have shape (P, 2)")
    _raise_if(len(cs) != 2, "atom_coords must be 2D")
    _raise_if(cs[1] != 3, "atom_coords must have shape (N, 3)")
    _raise_if(len(ts) != 1, "atom_types must be 1D")
    _raise_if(ts != (cs[0],), "atom_types must have shape (N,)")
    _raise_if(len(bs) != 2, "slice_z_bounds must be 2D")
    _raise_if(bs[1] != 2, "slice_z_bounds must have shape (S, 2)")
    _raise_if(len(vs) != 3, "atom_potentials must be 3D")
    _raise_if(ps[:2] != vs[1:], "probe_modes spatial shape must match atom_potentials")
    _checked_microscope(microscope)
    _checked_detector(detector)
    _checked_beam(probe_modes)
    _error_if(not _all_finite(probe_modes.modes), "probe_modes contain non-finite values")
    _error_if(not _all_finite(pos), "scan_positions_ang contain non-finite values")
    _error_if(not _all_finite(sample.atom_coords), "atom_coords contain non-finite values")
    zb = torch.as_tensor(sample.slice_z_bounds, dtype=torch.float64)
    _error_if(not _all_finite(zb), "slice_z_bounds contain non-finite values")
    _error_if(bool((zb[:, 1] - zb[:, 0] <= 0).any()), "slice_z_bounds thicknesses must be positive")
    _error_if(not _all_finite(sample.atom_potentials), "atom_potentials contain non-finite values")
    h, w = ps[0], ps[1]
    c = float(detector.real_space_calib_ang)
    t = torch.as_tensor(pos, dtype=torch.float64)
    _error_if(bool(((t[:, 0] < 0) | (t[:, 1] < 0) | (t[:, 0] >= h * c) | (t[:, 1] >= w * c)).any()),
              "scan_positions_ang must be within atom_potentials grid bounds")
    checked = create_atomic_slice_data(sample.atom_coords, sample.atom_types, sample.slice_z_bounds,
                                       sample.atom_potentials, sample.atom_mask)
    return stem4d_sharded(probe_modes, checked, microscope, detector, mesh)
