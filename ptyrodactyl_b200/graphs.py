"""CUDA-graph capture of fixed-shape multislice forwards.

A forward is a fixed sequence of a few thousand kernel launches (setup, then per
probe batch a ramp kernel and S + 2 passes). For a geometry that is run again
and again — a benchmark step, a serving request class, an iterative
reconstruction — :class:`GraphedForward` captures that sequence once into a CUDA
graph on static input/output buffers and replays it, so the host issues one
graph launch instead of thousands of kernel launches. Inputs are updated in place
(``copy_`` into :attr:`slices`, :attr:`modes`, :attr:`positions`...) between replays.
Each replay zeroes and then fills the device status words at the start of its
workspaces; :meth:`check` reads them after a replay.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib
from .simulations import check_windows, lane_batch, ms_params


class GraphedForward:
    """Captured ``ptyro_ms_forward`` on static device buffers.

    slices (F, F, S) float32, modes (n, n, M) complex64, weights (M,) float32,
    positions (P, 2) float64 (and optional windows (P, 2) int32) are kept by
    reference: write new inputs into them in place, then :meth:`replay`.

    ``lanes`` > 1 splits the probes into that many contiguous ranges, each run by
    its own forward on its own stream inside the same graph, so one range's passes
    fill the SMs that another range's pass leaves idle at its tail.
    """

    def __init__(self, slices: torch.Tensor, modes: torch.Tensor, weights: torch.Tensor, positions: torch.Tensor,
                 slice_thickness: float, voltage_kv: float, calib_ang: float,
                 shift_calib_ang: Optional[float] = None, batch: int = 0, tune: int = 0,
                 windows: Optional[torch.Tensor] = None, lanes: int = 1):
        self.lib = _lib.load()
        self.slices, self.modes, self.weights, self.positions, self.windows = slices, modes, weights, positions, windows
        dev = slices.device
        num_probes = positions.shape[0]
        n, f = check_windows(slices, modes, windows, num_probes)
        sc = calib_ang if shift_calib_ang is None else shift_calib_ang
        self.out = torch.empty((num_probes, n, n), dtype=torch.float32, device=dev)
        lanes = max(1, min(int(lanes), max(1, num_probes)))
        bounds = [num_probes * i // lanes for i in range(lanes + 1)]
        batch = lane_batch(n, modes.shape[2], lanes, batch)  # concurrent lanes share the L2 budget
        self.parts = []  # (lo, hi, params, workspace, bytes)
        for lo, hi in zip(bounds[:-1], bounds[1:]):
            prm = ms_params(n, slices.shape[2], modes.shape[2], hi - lo, voltage_kv, slice_thickness, calib_ang, sc,
                            slices.stride(), modes.stride(), batch, tune, f,
                            None if windows is None else windows[lo:hi])
            nbytes = self.lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
            if nbytes == 0:
                _lib.check(_lib.PTYRO_ERR_INVALID)
            self.parts.append((lo, hi, prm, torch.empty(nbytes, dtype=torch.uint8, device=dev), nbytes))
        # the first range's parameters and workspace (callers time single passes on them)
        self.prm, self.ws, self.ws_bytes = self.parts[0][2], self.parts[0][3], self.parts[0][4]
        self.streams = [torch.cuda.Stream(device=dev) for _ in self.parts] if lanes > 1 else []
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

    def _launch(self, part, stream: torch.cuda.Stream) -> None:
        lo, hi, prm, ws, nbytes = part
        rc = self.lib.ptyro_ms_forward(ctypes.byref(prm), self.slices.data_ptr(), self.modes.data_ptr(),
                                       self.weights.data_ptr(), self.positions[lo:hi].data_ptr(),
                                       self.out[lo:hi].data_ptr(), ws.data_ptr(), nbytes, stream.cuda_stream)
        _lib.check(rc)

    def _run(self, stream: torch.cuda.Stream) -> None:
        if not self.streams:
            self._launch(self.parts[0], stream)
            return
        for part, st in zip(self.parts, self.streams):  # fork
            st.wait_stream(stream)
            self._launch(part, st)
        for st in self.streams:  # join
            stream.wait_stream(st)

    def replay(self) -> torch.Tensor:
        """Run the captured forward on the current stream; returns the static output."""
        self.graph.replay()
        return self.out

    def status(self) -> int:
        """OR of the device status words the last replay left (waits for the replay)."""
        v = 0
        for part in self.parts:
            v |= int(part[3][:4].view(torch.int32).item())
        return v

    def check(self) -> None:
        """Raise ``DeviceStatusError`` if the last replay's kernels reported a failure."""
        v = self.status()
        if v:
            raise _lib.DeviceStatusError("graphed forward", v)
