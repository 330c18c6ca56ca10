"""Projected potentials of single atoms (src/ptyrodactyl/multislice/atom_potentials.py:588-681,
multislice/form_factors.py:132-439) on the device.

Coefficient tables (``data/``): the Lobato--Van Dyck parametrisation, five amplitude /
scale pairs per element for Z = 1..103 (I. Lobato and D. Van Dyck, Acta Cryst. A 70
(2014) 636-649, doi:10.1107/S205327331401643X; columns Z, element, a1..a5, b1..b5), and
Kirkland's three Lorentzian and three Gaussian pairs (E. J. Kirkland, Advanced Computing
in Electron Microscopy; one row per element, pairs interleaved a1, b1, ..., c3, d3).
Both are the tables the reference ships (``inout/luggage``).
"""

from __future__ import annotations

import os
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib
from .simulations import _device, _stream_ptr

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
_TABLES: dict = {}
PARAMETERIZATIONS = ("lobato", "kirkland")


def _table(name: str) -> np.ndarray:
    if name not in _TABLES:
        if name == "lobato":
            raw = np.loadtxt(os.path.join(_DATA, "lobato_van_dyck.csv"), delimiter=",", skiprows=1,
                             usecols=range(2, 12), dtype=np.float64)
        else:
            raw = np.loadtxt(os.path.join(_DATA, "kirkland_potentials.csv"), delimiter=",", dtype=np.float64)
        if raw.shape != (103, 10 if name == "lobato" else 12) or not np.all(np.isfinite(raw)):
            raise RuntimeError(f"the {name} coefficient table is malformed")
        _TABLES[name] = raw
    return _TABLES[name]


def _check_parameterization(parameterization: str) -> None:
    """form_factors.py:55-70."""
    if parameterization not in PARAMETERIZATIONS:
        raise ValueError("parameterization must be 'lobato' or 'kirkland'")


def _check_atom_no(atom_no) -> int:
    """form_factors.py:98-129."""
    if isinstance(atom_no, bool) or not float(atom_no).is_integer():
        raise ValueError("atom_no must be an integer between 1 and 103")
    z = int(atom_no)
    if z < 1 or z > 103:
        raise ValueError("atom_no must be between 1 and 103")
    return z


def lobato_parameters(atom_no) -> np.ndarray:
    """(a1..a5, b1..b5) of element ``atom_no`` (form_factors.py:132-164)."""
    return _table("lobato")[_check_atom_no(atom_no) - 1].copy()


def kirkland_parameters(atom_no) -> np.ndarray:
    """(a1, b1, a2, b2, a3, b3, c1, d1, c2, d2, c3, d3) of element ``atom_no``
    (form_factors.py:166-201; the first three pairs Lorentzian, the last three Gaussian)."""
    return _table("kirkland")[_check_atom_no(atom_no) - 1].copy()


def single_atom_potential(atom_no, pixel_size: float, grid_shape: Tuple[int, int], center_coords=None,
                          supersampling: int = 4, *, parameterization: str = "lobato",
                          device=None) -> torch.Tensor:
    """Projected potential (h, w) of one atom, volt-Angstrom, float64 on the device
    (atom_potentials.py:588-681): evaluated on a ``supersampling``-times finer grid
    (point k of an axis at (k - K/2) * pixel_size / supersampling, K = edge *
    supersampling) with the atom at ``center_coords`` = (x, y) in Angstrom (default
    the grid centre), then each pixel's supersampling^2 values averaged."""
    _check_parameterization(parameterization)
    coeffs = lobato_parameters(atom_no) if parameterization == "lobato" else kirkland_parameters(atom_no)
    h, w = int(grid_shape[0]), int(grid_shape[1])
    cx, cy = (0.0, 0.0) if center_coords is None else (float(center_coords[0]), float(center_coords[1]))
    dev = _device(device)
    out = torch.empty((h, w), dtype=torch.float64, device=dev)
    lib = _lib.load()
    with torch.cuda.device(dev):
        _lib.check(lib.ptyro_atom_potential(0 if parameterization == "lobato" else 1,
                                            coeffs.ctypes.data_as(_lib.ctypes.c_void_p), float(pixel_size), h, w,
                                            cx, cy, int(supersampling), out.data_ptr(), _stream_ptr(dev)))
    return out


def atom_lookup(atomic_numbers, pixel_size: float, grid_shape: Tuple[int, int], supersampling: int = 4,
                parameterization: str = "lobato", device=None) -> dict:
    """{Z: potential at the grid centre} for each element, as crystal_potential_slices
    builds its lookups (atom_potentials.py:1290-1312)."""
    return {int(z): single_atom_potential(int(z), pixel_size, grid_shape, (0.0, 0.0), supersampling,
                                          parameterization=parameterization, device=device)
            for z in sorted(set(int(v) for v in np.asarray(atomic_numbers).reshape(-1)))}


__all__ = ["single_atom_potential", "lobato_parameters", "kirkland_parameters", "atom_lookup", "PARAMETERIZATIONS"]
