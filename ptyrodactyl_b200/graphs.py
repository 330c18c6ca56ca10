"""CUDA-graph capture of fixed-shape multislice forwards.

A forward is a fixed sequence of a few thousand kernel launches (setup, then per
probe batch a ramp kernel and S + 2 passes). For a geometry that is run again
and again — a benchmark step, a serving request class, an iterative
reconstruction — :class:`GraphedForward` captures that sequence once into a CUDA
graph on static input/output buffers and replays it, so the host issues one
graph launch instead of thousands of kernel launches. Inputs are updated in place
(``copy_`` into :attr:`slices`, :attr:`modes`, :attr:`positions`...) between replays.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib
from .simulations import check_windows, ms_params


class GraphedForward:
    """Captured ``ptyro_ms_forward`` on static device buffers.

    slices (F, F, S) float32, modes (n, n, M) complex64, weights (M,) float32,
    positions (P, 2) float64 (and optional windows (P, 2) int32) are kept by
    reference: write new inputs into them in place, then :meth:`replay`.
    """

    def __init__(self, slices: torch.Tensor, modes: torch.Tensor, weights: torch.Tensor, positions: torch.Tensor,
                 slice_thickness: float, voltage_kv: float, calib_ang: float,
                 shift_calib_ang: Optional[float] = None, batch: int = 0, tune: int = 0,
                 windows: Optional[torch.Tensor] = None):
        self.lib = _lib.load()
        self.slices, self.modes, self.weights, self.positions, self.windows = slices, modes, weights, positions, windows
        dev = slices.device
        n, f = check_windows(slices, modes, windows, positions.shape[0])
        sc = calib_ang if shift_calib_ang is None else shift_calib_ang
        self.prm = ms_params(n, slices.shape[2], modes.shape[2], positions.shape[0], voltage_kv, slice_thickness,
                             calib_ang, sc, slices.stride(), modes.stride(), batch, tune, f, windows)
        self.ws_bytes = self.lib.ptyro_ms_workspace_bytes(ctypes.byref(self.prm))
        if self.ws_bytes == 0:
            _lib.check(_lib.PTYRO_ERR_INVALID)
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=dev)
        self.out = torch.empty((positions.shape[0], n, n), dtype=torch.float32, device=dev)
        self.launches_per_replay = 0
        # warm up outside capture (first launches set per-kernel attributes)
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            c0 = self.lib.ptyro_launch_count()
            self._run(side)
            self.launches_per_replay = int(self.lib.ptyro_launch_count() - c0)
        torch.cuda.current_stream(dev).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._run(torch.cuda.current_stream(dev))

    def _run(self, stream: torch.cuda.Stream) -> None:
        rc = self.lib.ptyro_ms_forward(ctypes.byref(self.prm), self.slices.data_ptr(), self.modes.data_ptr(),
                                       self.weights.data_ptr(), self.positions.data_ptr(), self.out.data_ptr(),
                                       self.ws.data_ptr(), self.ws_bytes, stream.cuda_stream)
        _lib.check(rc)

    def replay(self) -> torch.Tensor:
        """Run the captured forward on the current stream; returns the static output."""
        self.graph.replay()
        return self.out
