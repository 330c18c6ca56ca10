"""Potential slices of a crystal with sub-pixel atom placement on the device
(crystal_potential_slices, src/ptyrodactyl/multislice/atom_potentials.py:1364-1510).

The host restates the reference's bookkeeping — lattice repeats
(``_apply_repeats_or_return`` :1126-1241), slicing by z (``_slice_atoms`` :684-745),
the padded grid (``_compute_grid_dimensions`` :748-823) and the final crop — and the
device places every atom: per slice and atom type a structure factor (a product of
per-atom phase tables), times the spectrum of the type's projected potential, one
inverse FFT (``ptyro_place_atoms``; ``_process_all_slices`` :826-994).

Each element's projected potential comes from the Lobato or Kirkland parametrisation
(``single_atom_potential`` :588-681, evaluated on the device by ``elements.py``) on the
padded grid with the atom at its centre; callers may instead pass their own lookups
(``atom_potentials``: atomic number -> (H, W) array, the atom at the grid centre).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Mapping, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .simulations import SUPPORTED_EDGES, _device, _stream_ptr, _workspace
from .types import PotentialSlices, as_tensor, create_potential_slices


@dataclass(frozen=True)
class CrystalData:
    """Atoms of a crystal (types/crystal_types.py:84-124): positions (N, 3) in
    Angstrom, atomic numbers (N,), lattice vectors (3, 3) or None."""

    positions: np.ndarray
    atomic_numbers: np.ndarray
    lattice: Optional[np.ndarray] = None
    stress: Optional[np.ndarray] = None
    energy: Optional[float] = None
    comment: Optional[str] = None


def create_crystal_data(positions, atomic_numbers, lattice=None, stress=None, energy=None,
                        comment=None) -> CrystalData:
    """types/crystal_types.py:244-380, with the reference's messages."""
    pos = np.asarray(positions.cpu() if isinstance(positions, torch.Tensor) else positions, dtype=np.float64)
    nums = np.asarray(atomic_numbers.cpu() if isinstance(atomic_numbers, torch.Tensor) else atomic_numbers)
    if pos.ndim != 2:
        raise ValueError("positions must be 2D")
    if pos.shape[1] != 3:
        raise ValueError("positions must have shape (N, 3)")
    if nums.ndim != 1:
        raise ValueError("atomic_numbers must be 1D")
    if nums.shape[0] != pos.shape[0]:
        raise ValueError("atomic_numbers must have shape (N,)")
    lat = None if lattice is None else np.asarray(lattice, dtype=np.float64)
    if lat is not None and lat.shape != (3, 3):
        raise ValueError("lattice must have shape (3, 3)")
    st = None if stress is None else np.asarray(stress, dtype=np.float64)
    if st is not None and st.shape != (3, 3):
        raise ValueError("stress must have shape (3, 3)")
    if energy is not None and np.asarray(energy).shape != ():
        raise ValueError("energy must be a scalar")
    if not np.all(np.isfinite(pos)):
        raise ValueError("positions contain non-finite values")
    if np.any(nums < 0):
        raise ValueError("atomic_numbers must be non-negative")
    if lat is not None and not np.all(np.isfinite(lat)):
        raise ValueError("lattice contains non-finite values")
    return CrystalData(pos, nums.astype(np.int64), lat, st, None if energy is None else float(energy), comment)


def _apply_repeats(positions: np.ndarray, numbers: np.ndarray, lattice: np.ndarray, repeats) -> tuple:
    reps = [int(r) for r in np.asarray(repeats).reshape(-1)]
    if not any(r > 1 for r in reps):
        return positions, numbers
    ix, iy, iz = np.meshgrid(np.arange(reps[0]), np.arange(reps[1]), np.arange(reps[2]), indexing="ij")
    shifts = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=-1).astype(np.float64) @ lattice
    tiled = (positions[None, :, :] + shifts[:, None, :]).reshape(-1, 3)
    return tiled, np.tile(numbers, shifts.shape[0])


def _grid_dimensions(x, y, padding: float, pixel_size: float, height=None, width=None) -> tuple:
    x_min, y_min = float(np.min(x)) - padding, float(np.min(y)) - padding
    if height is not None and width is not None:
        return x_min, y_min, int(width), int(height)
    x_max, y_max = float(np.max(x)) + padding, float(np.max(y)) + padding
    w = int(np.ceil((x_max - x_min) / pixel_size))
    h = int(np.ceil((y_max - y_min) / pixel_size))
    crop = int(round(padding / pixel_size))
    return x_min, y_min, max(w, 2 * crop + 1), max(h, 2 * crop + 1)


def place_atoms(shift_y: np.ndarray, shift_x: np.ndarray, slice_index: np.ndarray, type_index: np.ndarray,
                lookup: torch.Tensor, num_slices: int, device=None) -> torch.Tensor:
    """Device placement: (n, n, num_slices) float32 slices from per-atom centre
    offsets in pixels, slice and type indices, and (T, n, n) lookup potentials."""
    lib = _lib.load()
    dev = _device(device)
    pots = as_tensor(lookup, torch.float32, dev).contiguous()
    num_types, n = pots.shape[0], pots.shape[1]
    keep = (slice_index >= 0) & (slice_index < num_slices)
    order = np.lexsort((type_index[keep], slice_index[keep]))  # by slice, then type; stable
    sl, ty = slice_index[keep][order], type_index[keep][order]
    sy = torch.as_tensor(np.ascontiguousarray(shift_y[keep][order], dtype=np.float64), device=dev)
    sx = torch.as_tensor(np.ascontiguousarray(shift_x[keep][order], dtype=np.float64), device=dev)
    groups = sl.astype(np.int64) * num_types + ty
    offsets = np.searchsorted(groups, np.arange(num_slices * num_types + 1), side="left").astype(np.int32)
    out = torch.empty((n, n, num_slices), dtype=torch.float32, device=dev)
    count = int(sy.numel())
    nbytes = lib.ptyro_place_atoms_workspace_bytes(n, num_types, count)
    ws = _workspace(nbytes, dev)
    _lib.check(lib.ptyro_place_atoms(n, count, num_types, num_slices, sy.data_ptr() if count else None,
                                     sx.data_ptr() if count else None,
                                     offsets.ctypes.data_as(ctypes.c_void_p), pots.data_ptr(), out.data_ptr(),
                                     *out.stride(), ws.data_ptr(), nbytes, _stream_ptr(dev)))
    return out  # the host offsets are read while the launches are enqueued


def crystal_potential_slices(crystal_data: CrystalData, pixel_size: float, slice_thickness: float = 1.0,
                             repeats=(1, 1, 1), padding: float = 4.0, supersampling: int = 4,
                             grid_shape: Optional[Tuple[int, int, int]] = None, *,
                             parameterization: str = "lobato",
                             atom_potentials: Optional[Mapping[int, object]] = None) -> PotentialSlices:
    """Potential slices of ``crystal_data`` (atom_potentials.py:1364-1510) on a padded
    grid, cropped by ``padding``. The padded grid must be square with a power-of-two
    edge in [16, 1024] (pass ``grid_shape``). Each element's lookup is its projected
    potential (``parameterization``, ``supersampling``) at the grid centre, or
    ``atom_potentials[Z]`` when given."""
    from .elements import _check_parameterization
    _check_parameterization(parameterization)
    if crystal_data.lattice is None:
        raise ValueError("CrystalData.lattice must not be None")
    positions, numbers = _apply_repeats(crystal_data.positions, crystal_data.atomic_numbers, crystal_data.lattice,
                                        repeats)
    z = positions[:, 2]
    slice_idx = np.floor((z - np.min(z)) / float(slice_thickness)).astype(np.int64)
    gh = gw = ns = None
    if grid_shape is not None:
        gh, gw, ns = (int(v) for v in grid_shape)
    x_min, y_min, width, height = _grid_dimensions(positions[:, 0], positions[:, 1], float(padding),
                                                   float(pixel_size), gh, gw)
    if height != width or height not in SUPPORTED_EDGES:
        raise ValueError(f"the padded grid must be square with an edge in {SUPPORTED_EDGES}, got ({height}, {width});"
                         " pass grid_shape")
    num_slices = ns if ns is not None else int(slice_idx.max()) + 1
    elements = sorted(set(int(v) for v in numbers))
    if atom_potentials is None:
        from .elements import atom_lookup
        atom_potentials = atom_lookup(elements, pixel_size, (height, width), supersampling, parameterization)
    missing = [e for e in elements if e not in atom_potentials]
    if missing:
        raise ValueError(f"atom_potentials has no entry for atomic numbers {missing}")
    lookup = np.stack([np.asarray(atom_potentials[e].cpu() if isinstance(atom_potentials[e], torch.Tensor)
                                  else atom_potentials[e], dtype=np.float32) for e in elements])
    if lookup.shape[1:] != (height, width):
        raise ValueError("atom_potentials must match the padded grid shape")
    type_idx = np.searchsorted(np.asarray(elements), numbers).astype(np.int64)
    shift_x = (positions[:, 0] - x_min) / float(pixel_size) - width / 2.0
    shift_y = (positions[:, 1] - y_min) / float(pixel_size) - height / 2.0
    slices = place_atoms(shift_y, shift_x, slice_idx, type_idx, torch.from_numpy(lookup), num_slices)
    crop = int(round(float(padding) / float(pixel_size)))
    cropped = slices[crop:height - crop, crop:width - crop, :]
    return create_potential_slices(cropped, slice_thickness, pixel_size)
