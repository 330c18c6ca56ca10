"""Public multislice API, call-compatible with ``ptyrodactyl.multislice``.

Each function keeps the signature and argument meaning of the reference
function it is named after (``src/ptyrodactyl/multislice/simulations.py``) and
runs on the GPU through the C-ABI of ``libptyro_b200.so``. There is no CPU
fallback: without CUDA or without the library every entry point raises.
"""

from __future__ import annotations

import ctypes
import math
import threading
from typing import Optional

import numpy as np
import torch

from . import _lib
from .types import (
    AtomicSliceData,
    CalibratedArray,
    DetectorConfig,
    MicroscopeConfig,
    PotentialSlices,
    ProbeModes,
    STEM4D,
    as_tensor,
    create_calibrated_array,
    create_probe_modes,
    create_stem4d,
)

# CODATA 2018 (types/constants.py:60-104)
H_PLANCK = 6.62607015e-34
HBAR = 1.054571817e-34
M_E = 9.1093837015e-31
E_CHARGE = 1.602176634e-19
C_LIGHT = 2.99792458e8
A_BOHR = 0.529177210903  # Angstrom
M0C2_EV = 510998.95
MOTT_BETHE_VOLT_ANGSTROM_SQ = 47.87801

SUPPORTED_EDGES = (16, 32, 64, 128, 256, 512, 1024)


def relativistic_wavelength_ang(voltage_kv: float) -> float:
    """Electron wavelength in Angstrom (types/constants.py:291-340)."""
    ev = float(voltage_kv) * 1000.0 * E_CHARGE
    return 1e10 * math.sqrt((H_PLANCK * H_PLANCK) * (C_LIGHT * C_LIGHT) /
                            (ev * (2.0 * M_E * (C_LIGHT * C_LIGHT) + ev)))


def interaction_sigma(voltage_kv: float) -> float:
    """sigma of transmission_func (simulations.py:150-157), rad / (V Angstrom)."""
    volt = float(voltage_kv) * 1000.0
    ev = E_CHARGE * volt
    einstein = M_E * (C_LIGHT * C_LIGHT)
    lam = relativistic_wavelength_ang(voltage_kv)
    return ((2 * math.pi / (lam * volt)) * (einstein + ev)) / ((2 * einstein) + ev)


def relativistic_mass(voltage_kv: float) -> float:
    """m = m_e (1 + e V / (m_e c^2)) in kg (types/constants.py:249-288)."""
    ev = float(voltage_kv) * 1000.0 * E_CHARGE
    return M_E * (1.0 + ev / (M_E * C_LIGHT * C_LIGHT))


def phase_interaction_parameter(voltage_kv: float) -> float:
    """sigma = 2 pi m e lambda / h^2 with the relativistic mass, in rad / (V Angstrom)
    (types/constants.py:181-246); the same quantity as ``interaction_sigma``."""
    lam_m = relativistic_wavelength_ang(voltage_kv) * 1e-10
    return 2.0 * math.pi * relativistic_mass(voltage_kv) * E_CHARGE * lam_m / (H_PLANCK * H_PLANCK) * 1e-10


def helmholtz_coupling(voltage_kv: float) -> float:
    """sigma_H = 2 m e / hbar^2 = 8 pi^2 m_0 e (1 + e U / (m_0 c^2)) / h^2, in
    1 / (V Angstrom^2) (types/constants.py:119-178); equals 2 k_0 sigma."""
    return 8.0 * math.pi ** 2 * relativistic_mass(voltage_kv) * E_CHARGE / (H_PLANCK * H_PLANCK) * 1e-20


def _device(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("ptyrodactyl_b200 needs a CUDA device (there is no CPU fallback)")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise RuntimeError("ptyrodactyl_b200 runs on CUDA devices only")
    return d


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _check_edge(h: int, w: int) -> int:
    if h != w:
        raise ValueError(f"grid must be square, got ({h}, {w})")
    if h not in SUPPORTED_EDGES:
        raise ValueError(f"grid edge must be one of {SUPPORTED_EDGES}, got {h}")
    return h


ANY_GRID_MAX = 4096  # height and width limit of the any-size path


def engine_grid(h: int, w: int) -> bool:
    """True for the pass engine's square power-of-two grids; every other height x
    width in [1, 4096] runs the any-size path (ptyro_gm_*)."""
    return int(h) == int(w) and int(h) in SUPPORTED_EDGES


def check_any_grid(slices: torch.Tensor, modes: torch.Tensor, windows: Optional[torch.Tensor] = None):
    """(H, W) of an any-size forward: the potential covers the beam's grid exactly."""
    h, w = int(modes.shape[0]), int(modes.shape[1])
    if not (1 <= h <= ANY_GRID_MAX and 1 <= w <= ANY_GRID_MAX):
        raise ValueError(f"grid height and width must be in [1, {ANY_GRID_MAX}], got ({h}, {w})")
    if windows is not None:
        raise ValueError(f"potential-field windows need a square grid with edge in {SUPPORTED_EDGES}, got ({h}, {w})")
    if tuple(slices.shape[:2]) != (h, w):
        raise ValueError(f"potential slices {tuple(slices.shape[:2])} must cover the beam grid ({h}, {w})")
    return h, w


def any_grid_params(slices: torch.Tensor, modes: torch.Tensor, num_probes: int, voltage_kv: float,
                    slice_thickness: float, calib_ang: float, shift_calib_ang: float, batch: int = 0,
                    accumulate: bool = False) -> _lib.MsParams:
    return ms_params(0, slices.shape[2], modes.shape[2], num_probes, voltage_kv, slice_thickness, calib_ang,
                     shift_calib_ang, slices.stride(), modes.stride(), batch, 0, 0, None,
                     _lib.PTYRO_FLAG_ACCUMULATE if accumulate else 0)


def run_forward_any(slices: torch.Tensor, slice_thickness: float, modes: torch.Tensor, weights: torch.Tensor,
                    positions: torch.Tensor, voltage_kv: float, calib_ang: float, shift_calib_ang: float,
                    out: Optional[torch.Tensor] = None, batch: int = 0, accumulate: bool = False,
                    status: Optional[torch.Tensor] = None, residuals: Optional[torch.Tensor] = None,
                    windows: Optional[torch.Tensor] = None) -> torch.Tensor:
    """``run_forward`` on any height x width grid (ptyro_gm_forward): the potential
    covers the beam's grid, no windows. ``residuals`` (ptyro_gm_residual_bytes) keeps
    the waves the any-size adjoint reads."""
    lib = _lib.load()
    dev = slices.device
    h, w = check_any_grid(slices, modes, windows)
    num_probes = positions.shape[0]
    prm = any_grid_params(slices, modes, num_probes, voltage_kv, slice_thickness, calib_ang, shift_calib_ang,
                          batch, accumulate)
    if out is None:
        out = (torch.zeros if accumulate else torch.empty)((num_probes, h, w), dtype=torch.float32, device=dev)
    if num_probes == 0:
        return out
    ws_bytes = lib.ptyro_gm_workspace_bytes(ctypes.byref(prm), h, w)
    if ws_bytes == 0:
        _lib.check(_lib.PTYRO_ERR_INVALID)
    ws = _workspace(ws_bytes, dev)
    with torch.cuda.device(dev):
        rc = lib.ptyro_gm_forward(ctypes.byref(prm), h, w, slices.data_ptr(), modes.data_ptr(), weights.data_ptr(),
                                  positions.data_ptr(), out.data_ptr(), _ptr(residuals), ws.data_ptr(), ws_bytes,
                                  _stream_ptr(dev))
    _lib.check(rc)
    _lib.gather_status(status, ws)
    return out


def _workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    # torch's caching allocator hands out 512-byte aligned blocks
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def ms_params(n: int, num_slices: int, num_modes: int, num_probes: int, voltage_kv: float,
              slice_thickness: float, calib_ang: float, shift_calib_ang: float,
              pot_strides=(0, 0, 0), mode_strides=(0, 0, 0), batch: int = 0, tune: int = 0,
              field_n: int = 0, windows: Optional[torch.Tensor] = None, flags: int = 0) -> _lib.MsParams:
    p = _lib.MsParams()
    p.flags = int(flags)
    p.n, p.num_slices, p.num_modes, p.num_probes, p.batch = n, num_slices, num_modes, num_probes, batch
    p.tune = tune
    p.field_n = 0 if field_n == n else int(field_n)
    p.windows = None if windows is None else windows.data_ptr()
    p.voltage_kv = float(voltage_kv)
    p.slice_thickness_ang = float(slice_thickness)
    p.calib_ang = float(calib_ang)
    p.shift_calib_ang = float(shift_calib_ang)
    p.pot_stride_y, p.pot_stride_x, p.pot_stride_s = (int(s) for s in pot_strides)
    p.mode_stride_y, p.mode_stride_x, p.mode_stride_m = (int(s) for s in mode_strides)
    return p


def check_windows(slices: torch.Tensor, modes: torch.Tensor, windows: Optional[torch.Tensor], num_probes: int):
    """Grid edge n (from the beam) and field edge F (from the potential)."""
    n = _check_edge(modes.shape[0], modes.shape[1])
    f = slices.shape[0]
    if slices.shape[0] != slices.shape[1]:
        raise ValueError(f"potential field must be square, got {tuple(slices.shape[:2])}")
    if f != n:
        if f < n or f & (f - 1) or f > 8192:
            raise ValueError(f"potential field edge must be a power of two in [{n}, 8192], got {f}")
    elif windows is None:
        return n, f
    if windows is not None:
        if windows.dtype != torch.int32 or tuple(windows.shape) != (num_probes, 2) or not windows.is_contiguous():
            raise ValueError("windows must be a contiguous (P, 2) int32 tensor")
        if windows.device != slices.device:
            raise ValueError("windows must be on the potential's device")
    return n, f


# Launch variant per grid edge measured fastest on B200 (ptyro_ms_params.tune bits:
# 1/2 three CTAs per SM per axis, 16 paired two-lines-per-thread steady passes,
# 64 eight warps per CTA, 128 direct column access, 256 half-paired lines of N2 = 2 N1,
# 2048 column blocks moved by TMA at 256^2 and 512^2, 4096 first and last slice
# passes paired at 256^2, 16384 interleaved transmission tables: line pairs at 256^2,
# line halves at 512^2, 32768 the wave-resident kernel at 128^2 for the forwards it
# applies to);
# the autotuner refines it.
DEFAULT_TUNE = {16: 147, 32: 147, 64: 147, 128: 32915, 256: 22739, 512: 18691, 1024: 0}


def default_tune(n: int) -> int:
    return DEFAULT_TUNE.get(int(n), 0)


_LANE_MIN_WAVE_BYTES = 256 << 20  # two lanes once the probes' waves span about four batches
# Wave slots in flight across all concurrent lanes. The engine's own batch keeps one
# forward's slots near 64 MiB, resident in the 126 MB L2; lanes running side by side
# share that budget, so the passes stay off DRAM (measured at 256^2, two lanes: 64
# probes per lane 3.47 M updates/s at 1965 MHz, 128 per lane 3.13 M/s, power-capped
# at 1785 MHz by the DRAM traffic).
L2_WAVE_BUDGET_BYTES = 64 << 20


def lane_batch(n: int, num_modes: int, lanes: int, batch: int = 0) -> int:
    """Probes per batch of one of ``lanes`` concurrent forwards: ``batch`` when given,
    else (several lanes, grids up to 256^2) the lane's share of ``L2_WAVE_BUDGET_BYTES``;
    0 leaves the choice to the engine. At 512^2 the engine's own batches measured faster
    (the 512^2 leg: 0.61 M updates/s with 32 probes per lane, 0.50 M with 16)."""
    if batch > 0 or lanes <= 1 or n > 256:
        return int(batch)
    return max(1, L2_WAVE_BUDGET_BYTES // int(lanes) // (8 * int(n) * int(n) * int(num_modes)))


def _side_streams(dev: torch.device, count: int) -> list:
    key = (dev.index, count)
    if key not in _STREAMS:
        _STREAMS[key] = [torch.cuda.Stream(device=dev) for _ in range(count)]
    return _STREAMS[key]


_STREAMS: dict = {}


def run_forward(slices: torch.Tensor, slice_thickness: float, modes: torch.Tensor, weights: torch.Tensor,
                positions: torch.Tensor, voltage_kv: float, calib_ang: float, shift_calib_ang: float,
                out: Optional[torch.Tensor] = None, batch: int = 0, plain: bool = False,
                tune: Optional[int] = None, windows: Optional[torch.Tensor] = None, accumulate: bool = False,
                lanes: int = 0, status: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Device-level forward: all tensors already on one CUDA device.

    slices (F, F, S) float32 (any strides), modes (n, n, M) complex64 (any strides),
    weights (M,) float32, positions (P, 2) float64 contiguous. F == n, or F > n with
    ``windows`` (P, 2) int32: probe p then reads the n x n window of the periodic
    field starting at windows[p]. Returns patterns (P, n, n) float32; with
    ``accumulate`` the intensities are added into ``out`` instead. ``lanes`` > 1
    runs contiguous probe ranges as concurrent forwards on side streams (0: two
    lanes when the probes' waves exceed 256 MiB); results do not depend on it.
    ``status`` (an int32 device word from ``_lib.new_status``) collects the call's
    device status bits asynchronously; nothing here synchronises, so the caller checks
    it (``_lib.check_status``) once it needs the results.
    """
    if not engine_grid(modes.shape[0], modes.shape[1]):
        return run_forward_any(slices, slice_thickness, modes, weights, positions, voltage_kv, calib_ang,
                               shift_calib_ang, out=out, batch=batch, accumulate=accumulate, status=status,
                               windows=windows)
    lib = _lib.load()
    dev = slices.device
    num_probes = positions.shape[0]
    n, f = check_windows(slices, modes, windows, num_probes)
    if tune is None:
        tune = default_tune(n)
    if lanes == 0:
        lanes = 2 if (not plain and num_probes * n * n * modes.shape[2] * 8 >= _LANE_MIN_WAVE_BYTES) else 1
    if lanes > 1 and num_probes >= lanes:
        if out is None:
            out = (torch.zeros if accumulate else torch.empty)((num_probes, n, n), dtype=torch.float32, device=dev)
        main = torch.cuda.current_stream(dev)
        bounds = [num_probes * i // lanes for i in range(lanes + 1)]
        streams = _side_streams(dev, lanes)
        # one status word per lane: the lanes run concurrently
        lane_status = [None if status is None else _lib.new_status(dev) for _ in streams]
        lb = lane_batch(n, modes.shape[2], lanes, batch)
        for (lo, hi), st, ls in zip(zip(bounds[:-1], bounds[1:]), streams, lane_status):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                run_forward(slices, slice_thickness, modes, weights, positions[lo:hi], voltage_kv, calib_ang,
                            shift_calib_ang, out=out[lo:hi], batch=lb, plain=plain, tune=tune,
                            windows=None if windows is None else windows[lo:hi], accumulate=accumulate, lanes=1,
                            status=ls)
        for st in streams:
            main.wait_stream(st)
        for ls in lane_status:
            if ls is not None:
                status.bitwise_or_(ls)
        return out
    prm = ms_params(n, slices.shape[2], modes.shape[2], num_probes, voltage_kv, slice_thickness,
                    calib_ang, shift_calib_ang, slices.stride(), modes.stride(), batch, tune, f, windows,
                    _lib.PTYRO_FLAG_ACCUMULATE if accumulate else 0)
    if out is None:
        out = (torch.zeros if accumulate else torch.empty)((num_probes, n, n), dtype=torch.float32, device=dev)
    if num_probes == 0:
        return out
    ws_bytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    if ws_bytes == 0:
        _lib.check(_lib.PTYRO_ERR_INVALID)
    ws = _workspace(ws_bytes, dev)
    fn = lib.ptyro_ms_forward_plain if plain else lib.ptyro_ms_forward
    with torch.cuda.device(dev):  # the engine launches on, and keeps per-device state for, the current device
        rc = fn(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(), weights.data_ptr(),
                positions.data_ptr(), out.data_ptr(), ws.data_ptr(), ws_bytes, _stream_ptr(dev))
    _lib.check(rc)
    if not plain:
        _lib.gather_status(status, ws)
    return out


def run_forward_to_host(slices: torch.Tensor, slice_thickness: float, modes: torch.Tensor, weights: torch.Tensor,
                        positions: torch.Tensor, voltage_kv: float, calib_ang: float, shift_calib_ang: float,
                        host_out: torch.Tensor, lanes: int = 2, tune: Optional[int] = None,
                        windows: Optional[torch.Tensor] = None,
                        status: Optional[torch.Tensor] = None) -> torch.Tensor:
    """``run_forward`` whose patterns land in a host tensor (pinned for overlap): the
    probes run as ``lanes`` contiguous ranges, each one forward on a compute stream of
    its own (``ptyro_ms_forward_to_host``) that copies every probe batch's patterns to
    the host on a copy stream of its own as soon as the batch is done, so the
    device-to-host transfer overlaps the remaining compute and only the last batch's
    copy is exposed."""
    dev = slices.device
    num_probes = positions.shape[0]
    any_grid = not engine_grid(modes.shape[0], modes.shape[1])
    if any_grid:
        h, w = check_any_grid(slices, modes, windows)
        f = h
    else:
        h, f = check_windows(slices, modes, windows, num_probes)
        w = h
    if tuple(host_out.shape) != (num_probes, h, w) or host_out.dtype != torch.float32:
        raise ValueError(f"host_out must be a float32 tensor of shape {(num_probes, h, w)}")
    if num_probes == 0:
        return host_out
    if any_grid:  # one forward, then one copy
        host_out.copy_(run_forward_any(slices, slice_thickness, modes, weights, positions, voltage_kv, calib_ang,
                                       shift_calib_ang, status=status), non_blocking=True)
        return host_out
    lib = _lib.load()
    if tune is None:
        tune = default_tune(h)
    dev_out = torch.empty((num_probes, h, w), dtype=torch.float32, device=dev)
    main = torch.cuda.current_stream(dev)
    lanes = max(1, min(int(lanes), num_probes))
    streams = _side_streams(dev, lanes)
    copies = _copy_streams(dev, lanes)
    bounds = [num_probes * i // lanes for i in range(lanes + 1)]
    lb = lane_batch(h, modes.shape[2], lanes)
    lane_status = [None if status is None else _lib.new_status(dev) for _ in streams]
    calls = []  # (params, workspace, bytes, lo, hi, compute stream, copy stream)
    for (lo, hi), st, cp in zip(zip(bounds[:-1], bounds[1:]), streams, copies):
        st.wait_stream(main)
        cp.wait_stream(main)
        prm = ms_params(h, slices.shape[2], modes.shape[2], hi - lo, voltage_kv, slice_thickness, calib_ang,
                        shift_calib_ang, slices.stride(), modes.stride(), lb, tune, f,
                        None if windows is None else windows[lo:hi])
        ws_bytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
        if ws_bytes == 0:
            _lib.check(_lib.PTYRO_ERR_INVALID)
        with torch.cuda.stream(st):
            ws = _workspace(ws_bytes, dev)  # allocated for the lane's stream
        calls.append((prm, ws, ws_bytes, lo, hi, st, cp))
    results = [None] * len(calls)

    def issue(i):
        prm, ws, ws_bytes, lo, hi, st, cp = calls[i]
        try:
            with torch.cuda.device(dev):
                rc = lib.ptyro_ms_forward_to_host(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(),
                                                  weights.data_ptr(), positions[lo:hi].data_ptr(),
                                                  dev_out[lo:hi].data_ptr(), host_out[lo:hi].data_ptr(),
                                                  ws.data_ptr(), ws_bytes, st.cuda_stream, cp.cuda_stream)
                # the library's error message is per thread
                results[i] = (rc, lib.ptyro_last_error().decode() if rc else "")
        except Exception as error:  # reported on the calling thread below
            results[i] = (_lib.PTYRO_ERR_CUDA, f"issuing lane {i}: {error!r}")

    # each lane's launches are issued from a host thread of its own (the call releases
    # the interpreter lock), so both lanes reach the GPU from the start
    threads = [threading.Thread(target=issue, args=(i,)) for i in range(1, len(calls))]
    for t in threads:
        t.start()
    issue(0)
    for t in threads:
        t.join()
    for rc, msg in results:
        if rc in (_lib.PTYRO_ERR_INVALID, _lib.PTYRO_ERR_UNSUPPORTED):
            raise ValueError(msg)
        if rc:
            raise _lib.PtyroError(rc, msg)
    for (prm, ws, ws_bytes, lo, hi, st, cp), ls in zip(calls, lane_status):
        with torch.cuda.stream(st):
            _lib.gather_status(ls, ws)  # one status word per lane: the lanes run concurrently
    for st in streams:
        main.wait_stream(st)
    for ls in lane_status:
        if ls is not None:
            status.bitwise_or_(ls)
    return host_out


def _copy_streams(dev: torch.device, count: int) -> list:
    key = ("copy", dev.index, count)
    if key not in _STREAMS:
        _STREAMS[key] = [torch.cuda.Stream(device=dev) for _ in range(count)]
    return _STREAMS[key]


def _needs_autodiff(*tensors) -> bool:
    """True when a reverse- or forward-mode derivative will be taken through the
    forward (requires_grad, a torch.func transform's wrapper, or a dual tensor)."""
    from torch.autograd import forward_ad
    for t in tensors:
        if t.requires_grad and torch.is_grad_enabled():
            return True
        if torch._C._functorch.is_functorch_wrapped_tensor(t) or forward_ad.unpack_dual(t).tangent is not None:
            return True
    return False


def _ensemble_weights(microscope: MicroscopeConfig) -> list:
    """The weight tensors of the microscope's ensemble axes (a derivative may be taken
    with respect to them)."""
    ens = microscope.ensemble
    return [d.weights for d in (ens.probe_modes, ens.position_jitter, ens.coherence) if d is not None]


def _beam_on(beam: ProbeModes, dev) -> tuple:
    modes = beam.modes if beam.modes.ndim == 3 else beam.modes[..., None]
    modes = as_tensor(modes, torch.complex64, dev)
    weights = as_tensor(beam.weights, torch.float32, dev).contiguous()
    return modes, weights


def stem_4d(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
            detector: DetectorConfig, *, out: Optional[torch.Tensor] = None) -> STEM4D:
    """4D-STEM patterns at every scan position (simulations.py:1330-1443).

    ``detector.scan_positions_px`` is used exactly as the reference uses it: passed
    unchanged as the shift of ``shift_beam_fourier``, whose frequency grid is in
    1/Angstrom, so each value acts as Angstrom; the returned ``scan_positions``
    field is ``positions * real_space_calib_ang`` as in the reference. ``data`` is a
    float32 CUDA tensor (P, H, W), or ``out`` when given: a CUDA tensor is written in
    place; a host tensor (pinned) receives the patterns chunk by chunk while the
    remaining probes compute. The call waits for its kernels and raises
    ``DeviceStatusError`` if they reported a failure (a bounded wait that gave up).
    """
    if detector.scan_positions_px is None:
        raise ValueError("detector.scan_positions_px is required")
    dev = _device(pot_slice.slices.device if pot_slice.slices.is_cuda else None)
    slices = as_tensor(pot_slice.slices, torch.float32, dev)
    if slices.ndim == 2:
        slices = slices[..., None]
    modes, weights = _beam_on(beam, dev)
    positions = as_tensor(detector.scan_positions_px, torch.float64, dev).reshape(-1, 2).contiguous()
    calib = min(float(pot_slice.calib), float(beam.calib))
    if not microscope.ensemble.is_empty():
        # per position, cbed_image's ensemble branch (simulations.py:1163-1193)
        if _needs_autodiff(slices, modes, positions, weights, *_ensemble_weights(microscope)):
            from .ensemble import ensemble_patterns_differentiable
            data = ensemble_patterns_differentiable(slices, pot_slice.slice_thickness, beam, microscope.ensemble,
                                                    modes, weights, microscope.voltage_kv, calib, positions,
                                                    detector.real_space_calib_ang)
        else:
            from .ensemble import ensemble_patterns
            data = ensemble_patterns(slices, pot_slice.slice_thickness, beam, microscope.ensemble,
                                     microscope.voltage_kv, calib, positions, detector.real_space_calib_ang)
    elif _needs_autodiff(slices, modes, positions, weights):
        # differentiable path: checkpointed forward + hand-written adjoint kernel
        from .autodiff import stem_4d_patterns
        data = stem_4d_patterns(slices, modes, weights, positions, pot_slice.slice_thickness,
                                microscope.voltage_kv, calib, detector.real_space_calib_ang)
    elif out is not None and not out.is_cuda:
        status = _lib.new_status(dev)
        data = run_forward_to_host(slices, pot_slice.slice_thickness, modes, weights, positions,
                                   microscope.voltage_kv, calib, detector.real_space_calib_ang, out, status=status)
        _lib.check_status(status, "stem_4d")
    else:
        status = _lib.new_status(dev)
        data = run_forward(slices, pot_slice.slice_thickness, modes, weights, positions,
                           microscope.voltage_kv, calib, detector.real_space_calib_ang, out=out, status=status)
        _lib.check_status(status, "stem_4d")
    if out is not None and data is not out:
        out.copy_(data)
        data = out
    fourier_calib = 1.0 / (modes.shape[0] * calib)
    scan_positions = detector.scan_positions_px.to(torch.float64) * detector.real_space_calib_ang
    return create_stem4d(data, detector.real_space_calib_ang, fourier_calib, scan_positions,
                         microscope.voltage_kv)


def stem_4d_windowed(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
                     detector: DetectorConfig, windows) -> STEM4D:
    """stem_4d where probe p sees the (n x n) window of a larger periodic potential
    field that starts at pixel ``windows[p] = (y, x)``; positions shift the probe
    inside its window as in ``stem_4d``. The tiled counterpart of the reference's
    ``crystal2stem4d_tiled`` (src/ptyrodactyl/workflows/stem_4d.py:553), which crops
    a tile of the sample around each position."""
    if detector.scan_positions_px is None:
        raise ValueError("detector.scan_positions_px is required")
    dev = _device(pot_slice.slices.device if pot_slice.slices.is_cuda else None)
    slices = as_tensor(pot_slice.slices, torch.float32, dev)
    modes, weights = _beam_on(beam, dev)
    positions = as_tensor(detector.scan_positions_px, torch.float64, dev).reshape(-1, 2).contiguous()
    win = as_tensor(windows, torch.int32, dev).reshape(-1, 2).contiguous()
    calib = min(float(pot_slice.calib), float(beam.calib))
    if _needs_autodiff(slices, modes, positions):
        from .autodiff import stem_4d_patterns
        data = stem_4d_patterns(slices, modes, weights, positions, pot_slice.slice_thickness,
                                microscope.voltage_kv, calib, detector.real_space_calib_ang, windows=win)
    else:
        status = _lib.new_status(dev)
        data = run_forward(slices, pot_slice.slice_thickness, modes, weights, positions, microscope.voltage_kv,
                           calib, detector.real_space_calib_ang, windows=win, status=status)
        _lib.check_status(status, "stem_4d_windowed")
    fourier_calib = 1.0 / (modes.shape[0] * calib)
    scan_positions = detector.scan_positions_px.to(torch.float64) * detector.real_space_calib_ang
    return create_stem4d(data, detector.real_space_calib_ang, fourier_calib, scan_positions, microscope.voltage_kv)


def stem_4d_frozen_phonon(pot_slices: list, beam: ProbeModes, microscope: MicroscopeConfig,
                          detector: DetectorConfig) -> STEM4D:
    """Mean of ``stem_4d`` over frozen-phonon configurations (one PotentialSlices per
    configuration, same geometry). Each configuration's intensities are added into
    the output by the pattern pass with the mode weights scaled by 1/configurations."""
    if not pot_slices:
        raise ValueError("at least one potential configuration is required")
    if detector.scan_positions_px is None:
        raise ValueError("detector.scan_positions_px is required")
    dev = _device(pot_slices[0].slices.device if pot_slices[0].slices.is_cuda else None)
    modes, weights = _beam_on(beam, dev)
    wscaled = (weights / len(pot_slices)).contiguous()
    positions = as_tensor(detector.scan_positions_px, torch.float64, dev).reshape(-1, 2).contiguous()
    n = modes.shape[0]
    out = torch.zeros((positions.shape[0], n, n), dtype=torch.float32, device=dev)
    calib = min(float(pot_slices[0].calib), float(beam.calib))
    status = _lib.new_status(dev)
    for ps in pot_slices:
        slices = as_tensor(ps.slices, torch.float32, dev)
        run_forward(slices, ps.slice_thickness, modes, wscaled, positions, microscope.voltage_kv, calib,
                    detector.real_space_calib_ang, out=out, accumulate=True, status=status)
    _lib.check_status(status, "stem_4d_frozen_phonon")
    fourier_calib = 1.0 / (n * calib)
    scan_positions = detector.scan_positions_px.to(torch.float64) * detector.real_space_calib_ang
    return create_stem4d(out, detector.real_space_calib_ang, fourier_calib, scan_positions, microscope.voltage_kv)


def slices_from_atoms(sample: AtomicSliceData, grid_shape, calib_ang: float, device=None) -> torch.Tensor:
    """Potential slices (H, W, S) float32 built on the device from atoms
    (_compute_slice_potential, multislice/parallelized.py:54-169)."""
    lib = _lib.load()
    dev = _device(device)
    h, w = int(grid_shape[0]), int(grid_shape[1])
    n = _check_edge(h, w)
    pots = as_tensor(sample.atom_potentials, torch.float32, dev).contiguous()
    if tuple(pots.shape[1:]) != (n, n):
        raise ValueError("atom_potentials must match the grid shape")
    coords = as_tensor(sample.atom_coords, torch.float64, dev).contiguous()
    types = sample.atom_types.to(dev, torch.int32).contiguous()
    bounds = as_tensor(sample.slice_z_bounds, torch.float64).cpu().contiguous()
    mask = None if sample.atom_mask is None else as_tensor(sample.atom_mask, torch.float32, dev).contiguous()
    S = bounds.shape[0]
    out = torch.empty((n, n, S), dtype=torch.float32, device=dev)
    nbytes = lib.ptyro_atom_slices_workspace_bytes(n, pots.shape[0])
    ws = _workspace(nbytes, dev)
    _lib.check(lib.ptyro_atom_slices(n, coords.shape[0], pots.shape[0], S, coords.data_ptr(), types.data_ptr(),
                                     bounds.data_ptr(), pots.data_ptr(), None if mask is None else mask.data_ptr(),
                                     float(calib_ang), out.data_ptr(), *out.stride(), ws.data_ptr(), nbytes,
                                     _stream_ptr(dev)))
    return out


def stem4d_sharded(probe_modes: ProbeModes, sample: AtomicSliceData, microscope: MicroscopeConfig,
                   detector: DetectorConfig, mesh=None) -> STEM4D:
    """Atom-backed 4D-STEM (multislice/parallelized.py:348-536): slices built on the
    device from atoms, positions in Angstrom (``detector.scan_positions_ang``), every
    calibration = ``detector.real_space_calib_ang``. ``mesh`` must be None: this engine
    runs on one GPU per process (shard scan positions across processes instead)."""
    if detector.scan_positions_ang is None:
        raise ValueError("detector.scan_positions_ang is required")
    if mesh is not None:
        raise NotImplementedError("device meshes are not supported; shard positions across processes")
    dev = _device()
    modes, weights = _beam_on(probe_modes, dev)
    n = modes.shape[0]
    calib = float(detector.real_space_calib_ang)
    slices = slices_from_atoms(sample, (n, n), calib, dev)
    bounds = as_tensor(sample.slice_z_bounds, torch.float64)
    thickness = float(bounds[0, 1] - bounds[0, 0])
    positions = as_tensor(detector.scan_positions_ang, torch.float64, dev).reshape(-1, 2).contiguous()
    status = _lib.new_status(dev)
    data = run_forward(slices, thickness, modes, weights, positions, microscope.voltage_kv, calib, calib,
                       status=status)
    _lib.check_status(status, "stem4d_sharded")
    return create_stem4d(data, calib, 1.0 / (n * calib), detector.scan_positions_ang.to(torch.float64),
                         microscope.voltage_kv)


def cbed_amplitude_from_atoms(beam, atom_coords, atom_types, slice_z_bounds, atom_potentials, voltage_kv,
                              calib_ang, atom_mask=None) -> torch.Tensor:
    """Detector-plane amplitudes (H, W, M) complex64 of the unshifted beam modes through
    slices built on the device from atoms (multislice/parallelized.py:174-261); every
    calibration is ``calib_ang`` and the slice thickness is that of the first z bound."""
    from .types import create_atomic_slice_data
    dev = _device()
    modes = as_tensor(beam, torch.complex64, dev)
    if modes.ndim == 2:
        modes = modes[..., None]
    sample = create_atomic_slice_data(atom_coords, atom_types, slice_z_bounds, atom_potentials, atom_mask)
    slices = slices_from_atoms(sample, tuple(modes.shape[:2]), float(calib_ang), dev)
    bounds = as_tensor(sample.slice_z_bounds, torch.float64)
    thickness = float(bounds[0, 1] - bounds[0, 0])
    return _amplitudes_at_origin(slices, thickness, modes.contiguous(), float(voltage_kv), float(calib_ang))


def cbed_image_from_atoms(beam, mode_distribution, atom_coords, atom_types, slice_z_bounds, atom_potentials,
                          voltage_kv, calib_ang, atom_mask=None) -> torch.Tensor:
    """CBED intensity (H, W) of the atom-backed amplitudes reduced over
    ``mode_distribution`` (sample = mode index) by apply_distribution
    (multislice/parallelized.py:264-347)."""
    from .reduce import apply_distribution
    amps = cbed_amplitude_from_atoms(beam, atom_coords, atom_types, slice_z_bounds, atom_potentials, voltage_kv,
                                     calib_ang, atom_mask)
    return apply_distribution(mode_distribution, lambda sample: amps[..., int(sample[0])])


def cbed_image(pot_slices: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig) -> CalibratedArray:
    """Single-position CBED intensity (simulations.py:1130-1233): the unshifted beam
    through the slices, sum_m w_m |fftshift(fft2(exit wave))|^2, or, when the
    microscope carries ensemble axes, the ensemble branch (:1163-1193)."""
    dev = _device(pot_slices.slices.device if pot_slices.slices.is_cuda else None)
    slices = as_tensor(pot_slices.slices, torch.float32, dev)
    if slices.ndim == 2:
        slices = slices[..., None]
    modes, weights = _beam_on(beam, dev)
    calib = min(float(pot_slices.calib), float(beam.calib))
    zero = torch.zeros((1, 2), dtype=torch.float64, device=dev)
    if not microscope.ensemble.is_empty():
        if _needs_autodiff(slices, modes, weights, *_ensemble_weights(microscope)):
            from .ensemble import ensemble_patterns_differentiable
            data = ensemble_patterns_differentiable(slices, pot_slices.slice_thickness, beam, microscope.ensemble,
                                                    modes, weights, microscope.voltage_kv, calib, zero, calib)[0]
        else:
            from .ensemble import ensemble_patterns
            data = ensemble_patterns(slices, pot_slices.slice_thickness, beam, microscope.ensemble,
                                     microscope.voltage_kv, calib, zero, calib)[0]
    elif _needs_autodiff(slices, modes, weights):
        # the same engine call at the one zero position, through the adjoint kernels
        from .autodiff import stem_4d_patterns
        data = stem_4d_patterns(slices, modes, weights, zero, pot_slices.slice_thickness, microscope.voltage_kv,
                                calib, calib)[0]
    else:
        status = _lib.new_status(dev)
        data = run_forward(slices, pot_slices.slice_thickness, modes, weights, zero,
                           microscope.voltage_kv, calib, calib, status=status)[0]
        _lib.check_status(status, "cbed_image")
    inv = 1.0 / (modes.shape[0] * calib)
    return create_calibrated_array(data, inv, inv, False)


def cbed_amplitude(pot_slices: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig) -> torch.Tensor:
    """Complex detector-plane amplitudes (H, W, M) of every beam mode at the probe's
    own place: fftshift(fft2(exit wave)) (simulations.py:606-679), complex64 CUDA."""
    dev = _device(pot_slices.slices.device if pot_slices.slices.is_cuda else None)
    slices = as_tensor(pot_slices.slices, torch.float32, dev)
    if slices.ndim == 2:
        slices = slices[..., None]
    modes, _ = _beam_on(beam, dev)
    calib = min(float(pot_slices.calib), float(beam.calib))
    return _amplitudes_at_origin(slices, pot_slices.slice_thickness, modes, microscope.voltage_kv, calib)


def _amplitudes_at_origin(slices: torch.Tensor, slice_thickness: float, modes: torch.Tensor, voltage_kv: float,
                          calib: float) -> torch.Tensor:
    """fftshifted far-field amplitudes (H, W, M) complex64 of the unshifted modes."""
    lib = _lib.load()
    dev = slices.device
    microscope_kv = float(voltage_kv)
    zero = torch.zeros((1, 2), dtype=torch.float64, device=dev)
    if not engine_grid(modes.shape[0], modes.shape[1]):
        # the far-field amplitude planes of the any-size forward's residuals, fftshifted
        h, w = check_any_grid(slices, modes)
        S, M = slices.shape[2], modes.shape[2]
        prm = any_grid_params(slices, modes, 1, microscope_kv, slice_thickness, calib, calib)
        res = torch.empty(lib.ptyro_gm_residual_bytes(ctypes.byref(prm), h, w) // 8, dtype=torch.complex64,
                          device=dev)
        status = _lib.new_status(dev)
        run_forward_any(slices, slice_thickness, modes, torch.ones(M, dtype=torch.float32, device=dev),
                        zero, microscope_kv, calib, calib, status=status, residuals=res)
        _lib.check_status(status, "cbed_amplitude")
        amps = res.view(M, S + 1, h, w)[:, S]
        return torch.roll(amps, shifts=(h // 2, w // 2), dims=(1, 2)).permute(1, 2, 0)
    n, f = check_windows(slices, modes, None, 1)
    prm = ms_params(n, slices.shape[2], modes.shape[2], 1, microscope_kv, slice_thickness, calib,
                    calib, slices.stride(), modes.stride(), 0, 0, f)
    amps = torch.empty((1, modes.shape[2], n, n), dtype=torch.complex64, device=dev)
    nbytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = _workspace(nbytes, dev)
    _lib.check(lib.ptyro_ms_amplitudes(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(), zero.data_ptr(),
                                       None, amps.data_ptr(), ws.data_ptr(), nbytes, _stream_ptr(dev)))
    return amps[0].permute(1, 2, 0)


# ----------------------------------------------------------------------------- building blocks
# The reference's public per-step functions, float64/complex128 torch on the input's
# device and differentiable like the reference's. The engine evaluates the same
# quantities inside its kernels (k_transmission, k_propagator, k_ramps); these are for
# callers who compose their own steps.


def transmission_func(pot_slice, voltage_kv) -> torch.Tensor:
    """exp(i sigma V) of a potential slice (simulations.py:107-161), complex128."""
    v = as_tensor(pot_slice, torch.float64)
    return torch.polar(torch.ones_like(v), interaction_sigma(float(voltage_kv)) * v)


def propagation_func(imsize_y: int, imsize_x: int, thickness_ang, voltage_kv, calib_ang,
                     device=None) -> torch.Tensor:
    """Fresnel propagator exp(-i pi lambda dz (qx^2 + qy^2)) on the fftfreq grid
    (simulations.py:164-226), complex128 (imsize_y, imsize_x)."""
    dev = torch.device("cpu") if device is None else torch.device(device)
    qy = torch.fft.fftfreq(int(imsize_y), d=float(calib_ang), dtype=torch.float64, device=dev)
    qx = torch.fft.fftfreq(int(imsize_x), d=float(calib_ang), dtype=torch.float64, device=dev)
    l_sq = qx[None, :] ** 2 + qy[:, None] ** 2
    phase = -math.pi * relativistic_wavelength_ang(float(voltage_kv)) * float(thickness_ang) * l_sq
    return torch.polar(torch.ones_like(phase), phase)


def fourier_coords(calibration, image_size) -> CalibratedArray:
    """Radial spatial frequencies of a centred-then-rolled grid (simulations.py:229-294):
    |q| in 1/Angstrom (h, w) float64 with the inverse calibrations."""
    size = np.asarray(image_size, dtype=np.int64).reshape(-1)
    cal = np.broadcast_to(np.asarray(calibration, dtype=np.float64), (2,))
    fov = size * cal
    ay = np.arange(-size[0] / 2, size[0] / 2, 1) / fov[0]
    ax = np.arange(-size[1] / 2, size[1] / 2, 1) / fov[1]
    ry, rx = np.roll(ay, int(size[0] // 2)), np.roll(ax, int(size[1] // 2))
    xx, yy = np.meshgrid(rx, ry)
    radius = torch.from_numpy(np.sqrt(yy * yy + xx * xx))
    return create_calibrated_array(radius, float(ay[1] - ay[0]), float(ax[1] - ax[0]), False)


def fourier_calib(real_space_calib, sizebeam) -> torch.Tensor:
    """1 / (size x calibration) per axis (simulations.py:297-331), float64 (2,)."""
    return 1.0 / (as_tensor(np.asarray(sizebeam, dtype=np.float64), torch.float64)
                  * as_tensor(real_space_calib, torch.float64))


def decompose_beam_to_modes(beam: CalibratedArray, num_modes: int, key, first_mode_weight: float = 0.6) -> ProbeModes:
    """Orthogonal modes that together keep the beam's intensity (simulations.py:
    1447-1536): the reduced QR factor of an (H W, M) complex normal matrix drawn with
    ``key`` (two JAX key words or an int seed, split into the real and imaginary
    draws), each column scaled by the beam's pixel amplitudes |beam|; weights
    (first_mode_weight, then the rest shared equally). Modes complex128 on the host,
    as the reference returns them; the engine reads them as complex64."""
    from . import prng
    data = as_tensor(beam.data_array, torch.complex128).detach().cpu().numpy()
    hh, ww = data.shape
    m = int(num_modes)
    k1, k2 = prng.split(key)
    draws = prng.normal(k1, (hh * ww, m)) + 1j * prng.normal(k2, (hh * ww, m))
    q, _ = np.linalg.qr(draws, mode="reduced")
    weights = np.full(m, (1.0 - float(first_mode_weight)) / (m - 1) if m > 1 else 0.0)
    weights[0] = float(first_mode_weight)
    modes = (q * np.sqrt(np.abs(data.reshape(-1)) ** 2)[:, None]).reshape(hh, ww, m)
    checked = create_probe_modes(modes, weights, beam.calib_y)
    return ProbeModes(torch.from_numpy(modes), checked.weights, checked.calib)


def shift_beam_fourier(beam, pos, calib_ang) -> torch.Tensor:
    """ifft2(fft2(beam) exp(-2 pi i (qy y + qx x))) per position (simulations.py:
    1238-1327): beam (H, W) or (H, W, M), pos (P, 2) -> complex128 (P, H, W, M)."""
    b = as_tensor(beam, torch.complex128)
    if b.ndim == 2:
        b = b[..., None]
    dev = b.device
    p = as_tensor(pos, torch.float64, dev).reshape(-1, 2)
    qy = torch.fft.fftfreq(b.shape[0], d=float(calib_ang), dtype=torch.float64, device=dev)
    qx = torch.fft.fftfreq(b.shape[1], d=float(calib_ang), dtype=torch.float64, device=dev)
    bk = torch.fft.fft2(b, dim=(0, 1))
    phase = -2.0 * math.pi * (qy[None, :, None] * p[:, 0, None, None] + qx[None, None, :] * p[:, 1, None, None])
    ramp = torch.polar(torch.ones_like(phase), phase)
    return torch.fft.ifft2(bk[None] * ramp[..., None], dim=(1, 2))


def aberration(fourier_coord, lambda_angstrom, defocus=0.0, c3=0.0, c5=0.0) -> torch.Tensor:
    """Aberration phase chi = 2 pi / lambda (C1 p^2 / 2 + 1e7 C3 p^4 / 4 + 1e7 C5 p^6 / 6),
    p = lambda |q| (simulations.py:434-498; the 1e7 factor makes the C3 and C5 fields act
    as mm). ``fourier_coord`` is |q| in 1/Angstrom (any shape); float64 on its device,
    differentiable in every argument given as a tensor. ``make_probe`` evaluates the
    same phase inside its aperture kernel."""
    q = as_tensor(fourier_coord, torch.float64)
    dev = q.device

    def t(v):
        return v.to(device=dev, dtype=torch.float64) if isinstance(v, torch.Tensor) else torch.tensor(
            float(v), dtype=torch.float64, device=dev)
    lam = t(lambda_angstrom)
    p = lam * q
    chi = (t(defocus) * p ** 2) / 2 + (t(c3) * 1e7 * p ** 4) / 4 + (t(c5) * 1e7 * p ** 6) / 6
    return (2 * math.pi * chi) / lam


def make_probe(microscope: MicroscopeConfig, detector: DetectorConfig) -> torch.Tensor:
    """Real-space probe from aperture and aberrations (simulations.py:334-431):
    complex64 (H, W) CUDA tensor, centred at (H/2, W/2), unnormalised."""
    if microscope.probe_shape is None:
        raise ValueError("microscope.probe_shape is required")
    h, w = (int(v) for v in microscope.probe_shape)
    lib = _lib.load()
    dev = _device()
    if not engine_grid(h, w):
        if not (1 <= h <= ANY_GRID_MAX and 1 <= w <= ANY_GRID_MAX):
            raise ValueError(f"probe_shape must be in [1, {ANY_GRID_MAX}]^2, got ({h}, {w})")
        probe = torch.empty((h, w), dtype=torch.complex64, device=dev)
        ws_bytes = lib.ptyro_gm_make_probe_workspace_bytes(h, w)
        ws = _workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            rc = lib.ptyro_gm_make_probe(h, w, microscope.voltage_kv, microscope.aperture_mrad,
                                         detector.probe_calibration_pm, microscope.defocus_ang, microscope.c3_ang,
                                         microscope.c5_ang, probe.data_ptr(), ws.data_ptr(), ws_bytes,
                                         _stream_ptr(dev))
        _lib.check(rc)
        return probe
    n = h
    probe = torch.empty((n, n), dtype=torch.complex64, device=dev)
    ws_bytes = lib.ptyro_fft_workspace_bytes(n)
    ws = _workspace(ws_bytes, dev)
    rc = lib.ptyro_make_probe(n, microscope.voltage_kv, microscope.aperture_mrad,
                              detector.probe_calibration_pm, microscope.defocus_ang, microscope.c3_ang,
                              microscope.c5_ang, probe.data_ptr(), ws.data_ptr(), ws_bytes, _stream_ptr(dev))
    _lib.check(rc)
    return probe


def fft2(x: torch.Tensor, inverse: bool = False) -> torch.Tensor:
    """numpy-convention fft2/ifft2 over the last two axes of a complex64 CUDA tensor."""
    lib = _lib.load()
    dev = _device(x.device if x.is_cuda else None)
    y = as_tensor(x, torch.complex64, dev).contiguous().clone()
    if not engine_grid(y.shape[-2], y.shape[-1]):
        h, w = int(y.shape[-2]), int(y.shape[-1])
        ws_bytes = lib.ptyro_gm_fft_workspace_bytes(h, w)
        if ws_bytes == 0:
            raise ValueError(f"fft2 height and width must be in [1, {ANY_GRID_MAX}], got ({h}, {w})")
        ws = _workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            rc = lib.ptyro_gm_fft2(h, w, y.numel() // (h * w) if h * w else 0, 1 if inverse else 0, y.data_ptr(),
                                   ws.data_ptr(), ws_bytes, _stream_ptr(dev))
        _lib.check(rc)
        return y
    n = _check_edge(y.shape[-2], y.shape[-1])
    count = y.numel() // (n * n)
    ws_bytes = lib.ptyro_fft_workspace_bytes(n)
    ws = _workspace(ws_bytes, dev)
    _lib.check(lib.ptyro_fft2(n, count, 1 if inverse else 0, y.data_ptr(), ws.data_ptr(), ws_bytes,
                              _stream_ptr(dev)))
    return y
