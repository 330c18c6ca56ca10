"""Reverse-mode differentiation of the multislice forward model.

The reference differentiates ``stem_4d`` with ``jax.value_and_grad``
(``src/ptyrodactyl/multislice/multislice_recon.py:1940``); reverse mode through
its ``lax.scan`` keeps every slice's wave of every probe. Here the forward
records only checkpoints (every ``ckpt_every`` slices) and the complex far-field
amplitude, and the hand-written adjoint kernel (``ptyro_ms_backward``) runs the
slice operator backwards for the forward wave and the adjoint together. This is
the analogue of a ``jax.custom_vjp`` rule: :class:`Stem4dFunction` is a
``torch.autograd.Function`` whose backward calls the adjoint kernel.

Gradient conventions: torch returns ``2 dL/dconj(z)`` for a complex input of a
real loss; the C-ABI returns JAX's convention ``conj(2 dL/dconj(z))``; this module
converts between them.
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np
import torch

from . import _lib
from .simulations import (
    _LANE_MIN_WAVE_BYTES,
    _side_streams,
    _stream_ptr,
    _workspace,
    any_grid_params,
    check_any_grid,
    check_windows,
    default_tune,
    engine_grid,
    lane_batch,
    ms_params,
    relativistic_wavelength_ang,
    run_forward_any,
)

DEFAULT_CKPT = 0  # 0: every slice when the residuals fit RESIDUAL_BUDGET_BYTES, else ceil(sqrt(S))
# The default forward keeps the wave at every slice when that costs at most this many
# bytes: the adjoint then carries only lambda (half the transform work of the lockstep
# adjoint, which rebuilds the forward wave between sparser checkpoints).
RESIDUAL_BUDGET_BYTES = 16 << 30


def _ckpt_for(num_slices: int, ckpt_every: int, n: int = 0, planes: int = 0) -> int:
    """Checkpoint spacing: ``ckpt_every`` if given, else 1 when the S + 1 residual planes
    of all ``planes`` (probe, mode) slots of an n x n grid fit the budget, else ceil(sqrt(S))."""
    if ckpt_every and ckpt_every > 0:
        return int(ckpt_every)
    if n and planes and (num_slices + 1) * planes * 8 * n * n <= RESIDUAL_BUDGET_BYTES:
        return 1
    return max(1, int(math.ceil(math.sqrt(num_slices))))


def _plain(t: Optional[torch.Tensor]) -> Optional[torch.Tensor]:
    """The tensor under any functorch wrappers (None stays None)."""
    while t is not None and torch._C._functorch.is_functorch_wrapped_tensor(t):
        t = torch._C._functorch.get_unwrapped(t)
    return t


class Stem4dFunction(torch.autograd.Function):
    """(patterns, residuals) = stem_4d(slices, modes) with a checkpointed adjoint
    backward and a tangent-kernel forward-mode rule.

    slices (H, W, S) float32 CUDA (any strides); modes (H, W, M) complex64 CUDA (any
    strides); weights (M,) float32; positions (P, 2) float64. Weights and positions
    are constants (no derivative). ``record`` makes the forward keep the slice
    checkpoints and far-field amplitudes the backward needs; a forward-mode-only
    evaluation (``torch.func.jvp``, dual tensors) skips them. The residuals are the
    second, non-differentiable output.
    """

    @staticmethod
    def forward(slices, modes, weights, positions, slice_thickness: float, voltage_kv: float, calib_ang: float,
                shift_calib_ang: float, ckpt_every: int = 0, batch: int = 0, tune: int = 0, windows=None,
                record: bool = True):
        lib = _lib.load()
        dev = slices.device
        S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
        if not engine_grid(modes.shape[0], modes.shape[1]):
            return Stem4dFunction._forward_any(lib, slices, modes, weights, positions, slice_thickness, voltage_kv,
                                               calib_ang, shift_calib_ang, batch, windows, record)
        n, f = check_windows(slices, modes, windows, P)
        k = _ckpt_for(S, ckpt_every, n, P * M)
        prm = ms_params(n, S, M, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, slices.stride(),
                        modes.stride(), batch, tune, f, windows)
        out = torch.empty((P, n, n), dtype=torch.float32, device=dev)
        nres = lib.ptyro_ms_residual_bytes(ctypes.byref(prm), k) // 4 if (P and record) else 0
        res = torch.empty(nres, dtype=torch.float32, device=dev)
        if P and record:
            with torch.cuda.device(dev):
                run_forward_ckpt(slices, modes, weights, positions, k, slice_thickness, voltage_kv, calib_ang,
                                 shift_calib_ang, batch, tune, windows, out, res)
        elif P:
            ws_bytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
            ws = _workspace(ws_bytes, dev)
            with torch.cuda.device(dev):
                Stem4dFunction._forward_call(lib, prm, k, record, slices, modes, weights, positions, out, res, ws,
                                             ws_bytes, dev)
            _lib.check_workspace_status(ws, "stem_4d forward")
        return out, res

    @staticmethod
    def _forward_any(lib, slices, modes, weights, positions, slice_thickness, voltage_kv, calib_ang,
                     shift_calib_ang, batch, windows, record):
        """Any height x width (ptyro_gm_forward): the residuals hold every slice's wave
        and the far-field amplitudes, the any-size adjoint's only input."""
        h, w = check_any_grid(slices, modes, windows)
        P = positions.shape[0]
        prm = any_grid_params(slices, modes, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, batch)
        nres = lib.ptyro_gm_residual_bytes(ctypes.byref(prm), h, w) // 4 if (P and record) else 0
        res = torch.empty(nres, dtype=torch.float32, device=slices.device)
        status = _lib.new_status(slices.device)
        out = run_forward_any(slices, slice_thickness, modes, weights, positions, voltage_kv, calib_ang,
                              shift_calib_ang, batch=batch, status=status, residuals=res if nres else None)
        _lib.check_status(status, "stem_4d forward")
        return out, res

    @staticmethod
    def _forward_call(lib, prm, k, record, slices, modes, weights, positions, out, res, ws, ws_bytes, dev):
        if record:
            rc = lib.ptyro_ms_forward_ckpt(ctypes.byref(prm), k, slices.data_ptr(), modes.data_ptr(),
                                           weights.data_ptr(), positions.data_ptr(), out.data_ptr(),
                                           res.data_ptr(), ws.data_ptr(), ws_bytes, _stream_ptr(dev))
        else:
            rc = lib.ptyro_ms_forward(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(),
                                      weights.data_ptr(), positions.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                      ws_bytes, _stream_ptr(dev))
        _lib.check(rc)

    @staticmethod
    def setup_context(ctx, inputs, output):
        (slices, modes, weights, positions, slice_thickness, voltage_kv, calib_ang, shift_calib_ang, ckpt_every,
         batch, tune, windows, record) = inputs
        _, res = output
        ctx.mark_non_differentiable(res)
        ctx.save_for_backward(slices, modes, weights, positions, res, windows)
        ctx.save_for_forward(slices, modes, weights, positions, windows)
        n = modes.shape[0]
        ctx.any_grid = not engine_grid(modes.shape[0], modes.shape[1])
        ctx.cfg = (slice_thickness, voltage_kv, calib_ang, shift_calib_ang,
                   _ckpt_for(slices.shape[2], ckpt_every, n, positions.shape[0] * modes.shape[2]),
                   batch, tune, n, slices.shape[0], record)

    @staticmethod
    def backward(ctx, grad_out, grad_res):
        if not ctx.cfg[-1]:
            raise RuntimeError("stem_4d was evaluated without residuals (record=False); no backward")
        # under torch.func the rule sees functorch wrappers; the kernels need storage
        saved = [_plain(t) for t in ctx.saved_tensors]
        with torch._C._DisableFuncTorch(), torch.cuda.device(saved[0].device):
            g_slices, g_modes, g_pos = Stem4dFunction._adjoint(ctx, saved, _plain(grad_out))
            g_w = Stem4dFunction._weight_grad(ctx, saved, _plain(grad_out)) if ctx.needs_input_grad[2] else None
        return (g_slices if ctx.needs_input_grad[0] else None, g_modes if ctx.needs_input_grad[1] else None,
                g_w, g_pos, None, None, None, None, None, None, None, None, None)

    @staticmethod
    def _weight_grad(ctx, saved, grad_out):
        """dL/dw_m = sum_p sum_k dL/dI_p(k) |A_pm(k)|^2 from the stored far-field amplitudes
        (ptyro_ms_weight_grad), in the weights' dtype."""
        slices, modes, weights, positions, res, windows = saved
        slice_thickness, voltage_kv, calib_ang, shift_calib_ang, k, batch, tune, n, f, record = ctx.cfg
        lib = _lib.load()
        dev = slices.device
        S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
        out = torch.empty(M, dtype=torch.float64, device=dev)
        g = grad_out.to(torch.float32).contiguous()
        if ctx.any_grid:
            h, w = modes.shape[0], modes.shape[1]
            prm = any_grid_params(slices, modes, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, batch)
            nbytes = lib.ptyro_gm_weight_grad_workspace_bytes(ctypes.byref(prm), h, w)
            ws = _workspace(nbytes, dev)
            _lib.check(lib.ptyro_gm_weight_grad(ctypes.byref(prm), h, w, res.data_ptr(), g.data_ptr(),
                                                out.data_ptr(), ws.data_ptr(), nbytes, _stream_ptr(dev)))
            return out.to(weights.dtype)
        prm = ms_params(n, S, M, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, slices.stride(),
                        modes.stride(), batch, tune, f, windows)
        nbytes = lib.ptyro_ms_weight_grad_workspace_bytes(ctypes.byref(prm))
        ws = _workspace(nbytes, dev)
        _lib.check(lib.ptyro_ms_weight_grad(ctypes.byref(prm), k, res.data_ptr(), g.data_ptr(), out.data_ptr(),
                                            ws.data_ptr(), nbytes, _stream_ptr(dev)))
        return out.to(weights.dtype)

    @staticmethod
    def _adjoint(ctx, saved, grad_out):
        slices, modes, weights, positions, res, windows = saved
        slice_thickness, voltage_kv, calib_ang, shift_calib_ang, k, batch, tune, n, f, record = ctx.cfg
        lib = _lib.load()
        dev = slices.device
        S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
        g_slices = torch.empty_strided(slices.shape, slices.stride(), dtype=torch.float32, device=dev)
        g_modes = torch.empty_strided(modes.shape, modes.stride(), dtype=torch.complex64, device=dev)
        g_pos = torch.zeros((P, 2), dtype=torch.float64, device=dev) if ctx.needs_input_grad[3] else None
        if P == 0:
            g_slices.zero_()
            g_modes.zero_()
        elif ctx.any_grid:
            Stem4dFunction._adjoint_any(lib, slices, modes, weights, positions, res, grad_out, slice_thickness,
                                        voltage_kv, calib_ang, shift_calib_ang, batch, g_slices, g_modes, g_pos)
        else:
            run_backward(slices, modes, weights, positions, res, grad_out, k, slice_thickness, voltage_kv, calib_ang,
                         shift_calib_ang, batch, tune, windows, g_slices, g_modes, g_pos)
        # the C-ABI gives JAX's convention conj(2 dL/dconj); torch wants 2 dL/dconj
        return g_slices, g_modes.conj().resolve_conj(), g_pos

    @staticmethod
    def _adjoint_any(lib, slices, modes, weights, positions, res, grad_out, slice_thickness, voltage_kv, calib_ang,
                     shift_calib_ang, batch, g_slices, g_modes, g_pos):
        """ptyro_gm_backward: dL/dV, the modes' gradient (JAX's convention) and, when
        g_pos is given, dL/d(positions), from the any-size forward's residuals."""
        dev = slices.device
        h, w = modes.shape[0], modes.shape[1]
        P = positions.shape[0]
        prm = any_grid_params(slices, modes, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, batch)
        g = grad_out.to(torch.float32).contiguous()
        ws_bytes = lib.ptyro_gm_backward_workspace_bytes(ctypes.byref(prm), h, w)
        if ws_bytes == 0:
            _lib.check(_lib.PTYRO_ERR_INVALID)
        ws = _workspace(ws_bytes, dev)
        _lib.check(lib.ptyro_gm_backward(ctypes.byref(prm), h, w, slices.data_ptr(), modes.data_ptr(),
                                         weights.data_ptr(), positions.data_ptr(), res.data_ptr(), g.data_ptr(),
                                         g_slices.data_ptr(), g_modes.data_ptr(),
                                         None if g_pos is None else g_pos.data_ptr(), ws.data_ptr(), ws_bytes,
                                         _stream_ptr(dev)))
        _lib.check_workspace_status(ws, "stem_4d backward")

    @staticmethod
    def jvp(ctx, t_slices, t_modes, t_weights, t_positions, *rest):
        # under torch.func the rule sees functorch wrappers; the kernels need storage
        slices, modes, weights, positions, windows = (_plain(t) for t in ctx.saved_tensors)
        t_slices, t_modes, t_weights, t_positions = (_plain(t) for t in (t_slices, t_modes, t_weights, t_positions))
        slice_thickness, voltage_kv, calib_ang, shift_calib_ang, k, batch, tune, n, f, record = ctx.cfg
        # torch.func.jvp hands zero tangents to the inputs it does not differentiate
        moved = t_positions is not None and bool(t_positions.any())
        with torch._C._DisableFuncTorch():  # buffers made here must be plain tensors
            p_tangent = _position_tangent(slices, modes, weights, positions, t_positions, slice_thickness,
                                          voltage_kv, calib_ang, shift_calib_ang, batch, windows) if moved else None
            if t_weights is not None and bool(t_weights.any()):
                # the patterns are linear in the weights: their tangent is the forward with
                # the tangent weights, added to the potential's and modes' tangent below
                from .simulations import run_forward
                w_tangent = run_forward(slices, slice_thickness, modes, t_weights.to(torch.float32).contiguous(),
                                        positions, voltage_kv, calib_ang, shift_calib_ang, batch=batch,
                                        windows=windows)
            else:
                w_tangent = None
            _, tangent = jvp(slices, modes, weights, positions, t_slices, t_modes, slice_thickness, voltage_kv,
                             calib_ang, shift_calib_ang, batch=batch, windows=windows, want_patterns=False)
        if w_tangent is not None:
            tangent = tangent + w_tangent
        if p_tangent is not None:
            tangent = tangent + p_tangent
        return tangent, None


def _position_tangent(slices, modes, weights, positions, t_positions, slice_thickness, voltage_kv, calib_ang,
                      shift_calib_ang, batch, windows) -> torch.Tensor:
    """dI along scan-position tangents (P, 2). Probe p's first wave is
    ifft2(fft2(beam) R_p) with R_p = exp(-2 pi i (qy y_p + qx x_p)) (shift_beam_fourier,
    simulations.py:1236-1327), so d psi_p / dy_p = shift_p(ifft2(fft2(beam) (-2 pi i qy))):
    the tangent kernel with that fixed tangent beam, once per axis, gives every
    probe's derivative along its own y (x), and dI = dy_p dI/dy_p + dx_p dI/dx_p."""
    from .simulations import fft2
    dev = modes.device
    h, w = int(modes.shape[0]), int(modes.shape[1])
    spectra = fft2(modes.permute(2, 0, 1).contiguous())  # (M, H, W)
    qy = np.fft.fftfreq(h, d=float(shift_calib_ang))
    qx = np.fft.fftfreq(w, d=float(shift_calib_ang))
    out = None
    for c, q in enumerate((np.broadcast_to(qy[:, None], (h, w)), np.broadcast_to(qx[None, :], (h, w)))):
        factor = torch.as_tensor((-2j * np.pi * q).astype(np.complex64), device=dev)
        d_modes = fft2(spectra * factor, inverse=True).permute(1, 2, 0).contiguous()
        _, tan = jvp(slices, modes, weights, positions, None, d_modes, slice_thickness, voltage_kv, calib_ang,
                     shift_calib_ang, batch=batch, windows=windows, want_patterns=False)
        part = t_positions[:, c].to(device=dev, dtype=torch.float32)[:, None, None] * tan
        out = part if out is None else out + part
    return out


def _lanes_for(lib, P: int, n: int, S: int, M: int, k: int, lanes: int, prm_full, residuals) -> tuple:
    """(lanes, residual bytes per probe): two lanes when the probes' waves exceed
    256 MiB (as the forward), one when the residuals are not the probe-major layout the
    split assumes."""
    if lanes == 0:
        lanes = 2 if P * n * n * M * 8 >= _LANE_MIN_WAVE_BYTES else 1
    lanes = max(1, min(int(lanes), P))
    per_probe = M * ((S + k - 1) // k + 1) * n * n * 8
    if lanes > 1 and (lib.ptyro_ms_residual_bytes(ctypes.byref(prm_full), k) != P * per_probe
                      or residuals.numel() * residuals.element_size() < P * per_probe):
        lanes = 1
    return lanes, per_probe


def run_forward_ckpt(slices: torch.Tensor, modes: torch.Tensor, weights: torch.Tensor, positions: torch.Tensor,
                     ckpt_every: int, slice_thickness: float, voltage_kv: float, calib_ang: float,
                     shift_calib_ang: float, batch: int, tune: int, windows: Optional[torch.Tensor],
                     out: torch.Tensor, residuals: torch.Tensor, lanes: int = 0) -> None:
    """The residual-recording forward (ptyro_ms_forward_ckpt) into ``out`` (P, n, n) and
    ``residuals`` (ptyro_ms_residual_bytes); ``lanes`` > 1 runs contiguous probe ranges
    concurrently on side streams, each writing its own (probe-major) residual range, as
    ``run_backward`` reads them. The results do not depend on the lane count."""
    lib = _lib.load()
    dev = slices.device
    S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
    n, f = check_windows(slices, modes, windows, P)
    k = int(ckpt_every)
    full = ms_params(n, S, M, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, slices.stride(),
                     modes.stride(), batch, tune, f, windows)
    lanes, per_probe = _lanes_for(lib, P, n, S, M, k, lanes, full, residuals)
    main = torch.cuda.current_stream(dev)
    bounds = [P * i // lanes for i in range(lanes + 1)]
    streams = [main] if lanes == 1 else _side_streams(dev, lanes)
    lb = batch if lanes == 1 else lane_batch(n, M, lanes, batch)
    keep = []
    for (lo, hi), st in zip(zip(bounds[:-1], bounds[1:]), streams):
        win = None if windows is None else windows[lo:hi].contiguous()
        prm = full if lanes == 1 else ms_params(n, S, M, hi - lo, voltage_kv, slice_thickness, calib_ang,
                                                 shift_calib_ang, slices.stride(), modes.stride(), lb, tune, f, win)
        ws_bytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
        ws = _workspace(ws_bytes, dev)
        if st is not main:
            st.wait_stream(main)
        with torch.cuda.stream(st):
            _lib.check(lib.ptyro_ms_forward_ckpt(ctypes.byref(prm), k, slices.data_ptr(), modes.data_ptr(),
                                                 weights.data_ptr(), positions[lo:hi].data_ptr(),
                                                 out[lo:hi].data_ptr(), residuals.data_ptr() + lo * per_probe,
                                                 ws.data_ptr(), ws_bytes, _stream_ptr(dev)))
        if st is not main:
            for t in (ws,) + (() if win is None else (win,)):
                t.record_stream(st)
        keep.append(ws)
    for st in streams:
        if st is not main:
            main.wait_stream(st)
    for ws in keep:
        _lib.check_workspace_status(ws, "stem_4d forward")


def _backward_call(lib, prm, k, slices, modes, weights, positions, res_ptr, g, g_slices, g_modes, g_pos, ws,
                   ws_bytes, stream_ptr):
    if g_pos is None:
        _lib.check(lib.ptyro_ms_backward(ctypes.byref(prm), k, slices.data_ptr(), weights.data_ptr(),
                                         positions.data_ptr(), res_ptr, g.data_ptr(), g_slices.data_ptr(),
                                         g_modes.data_ptr(), ws.data_ptr(), ws_bytes, stream_ptr))
    else:
        _lib.check(lib.ptyro_ms_backward_positions(ctypes.byref(prm), k, slices.data_ptr(), modes.data_ptr(),
                                                   weights.data_ptr(), positions.data_ptr(), res_ptr, g.data_ptr(),
                                                   g_slices.data_ptr(), g_modes.data_ptr(), g_pos.data_ptr(),
                                                   ws.data_ptr(), ws_bytes, stream_ptr))


def run_backward(slices: torch.Tensor, modes: torch.Tensor, weights: torch.Tensor, positions: torch.Tensor,
                 residuals: torch.Tensor, grad_patterns: torch.Tensor, ckpt_every: int, slice_thickness: float,
                 voltage_kv: float, calib_ang: float, shift_calib_ang: float, batch: int, tune: int,
                 windows: Optional[torch.Tensor], g_slices: torch.Tensor, g_modes: torch.Tensor,
                 g_pos: Optional[torch.Tensor] = None, lanes: int = 0) -> None:
    """The engine's adjoint (ptyro_ms_backward, or _positions with ``g_pos``) over the
    residuals a ptyro_ms_forward_ckpt of the same probes recorded, into g_slices (the
    slices' strides) and g_modes (JAX's convention). ``lanes`` > 1 runs contiguous probe
    ranges as concurrent adjoints on side streams, each over its own residual range
    (the residuals are probe-major) with the lane's share of the L2 wave budget, their
    dL/dV and dL/dmodes added in lane order afterwards (0: two lanes when the probes'
    waves exceed 256 MiB, as the forward). The sums are deterministic for a given lane
    count; different lane counts agree to float32 rounding."""
    lib = _lib.load()
    dev = slices.device
    S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
    n, f = check_windows(slices, modes, windows, P)
    g = grad_patterns.to(torch.float32).contiguous()
    k = int(ckpt_every)
    full = ms_params(n, S, M, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, slices.stride(),
                     modes.stride(), batch, tune, f, windows)
    lanes, per_probe = _lanes_for(lib, P, n, S, M, k, lanes, full, residuals)
    if lanes == 1:
        prm = ms_params(n, S, M, P, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, slices.stride(),
                        modes.stride(), batch, tune, f, windows)
        ws_bytes = lib.ptyro_ms_backward_workspace_bytes(ctypes.byref(prm))
        ws = _workspace(ws_bytes, dev)
        _backward_call(lib, prm, k, slices, modes, weights, positions, residuals.data_ptr(), g, g_slices, g_modes,
                       g_pos, ws, ws_bytes, _stream_ptr(dev))
        _lib.check_workspace_status(ws, "stem_4d backward")
        return
    main = torch.cuda.current_stream(dev)
    bounds = [P * i // lanes for i in range(lanes + 1)]
    streams = _side_streams(dev, lanes)
    lb = lane_batch(n, M, lanes, batch)
    outs = [(g_slices, g_modes)] + [(torch.empty_strided(g_slices.shape, g_slices.stride(), dtype=g_slices.dtype,
                                                         device=dev),
                                     torch.empty_strided(g_modes.shape, g_modes.stride(), dtype=g_modes.dtype,
                                                         device=dev)) for _ in range(lanes - 1)]
    keep = []
    for (lo, hi), st, (gs, gm) in zip(zip(bounds[:-1], bounds[1:]), streams, outs):
        win = None if windows is None else windows[lo:hi].contiguous()
        prm = ms_params(n, S, M, hi - lo, voltage_kv, slice_thickness, calib_ang, shift_calib_ang, slices.stride(),
                        modes.stride(), lb, tune, f, win)
        ws_bytes = lib.ptyro_ms_backward_workspace_bytes(ctypes.byref(prm))
        ws = _workspace(ws_bytes, dev)
        st.wait_stream(main)
        with torch.cuda.stream(st):
            _backward_call(lib, prm, k, slices, modes, weights, positions[lo:hi],
                           residuals.data_ptr() + lo * per_probe, g[lo:hi], gs, gm,
                           None if g_pos is None else g_pos[lo:hi], ws, ws_bytes, _stream_ptr(dev))
        for t in (ws, gs, gm) + (() if win is None else (win,)):
            t.record_stream(st)
        keep.append(ws)
    for st in streams:
        main.wait_stream(st)
    for gs, gm in outs[1:]:
        g_slices.add_(gs)
        g_modes.add_(gm)
    for ws in keep:
        _lib.check_workspace_status(ws, "stem_4d backward")


def stem_4d_patterns(slices: torch.Tensor, modes: torch.Tensor, weights: torch.Tensor, positions: torch.Tensor,
                     slice_thickness: float, voltage_kv: float, calib_ang: float,
                     shift_calib_ang: Optional[float] = None, ckpt_every: int = DEFAULT_CKPT,
                     batch: int = 0, tune: Optional[int] = None,
                     windows: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Differentiable patterns (P, n, n) of the forward model (device tensors); with
    ``windows`` the potential is a larger periodic field (see ``run_forward``).
    Reverse mode (``backward``, ``torch.func.grad/vjp``) and forward mode
    (``torch.func.jvp``, dual tensors) both run hand-written kernels."""
    record = bool(slices.requires_grad or modes.requires_grad or positions.requires_grad or weights.requires_grad) \
        and torch.is_grad_enabled()
    return Stem4dFunction.apply(slices, modes, weights, positions, float(slice_thickness), float(voltage_kv),
                                float(calib_ang), float(calib_ang if shift_calib_ang is None else shift_calib_ang),
                                int(ckpt_every), int(batch), int(default_tune(modes.shape[0]) if tune is None else tune),
                                windows, record)[0]


def _like(t: Optional[torch.Tensor], primal: torch.Tensor, dtype) -> Optional[torch.Tensor]:
    """The tangent with the primal's strides (the kernels read both with one set)."""
    if t is None:
        return None
    t = t.to(device=primal.device, dtype=dtype)
    if t.shape != primal.shape:
        raise ValueError(f"tangent shape {tuple(t.shape)} does not match {tuple(primal.shape)}")
    if t.stride() == primal.stride():
        return t
    return torch.empty_strided(primal.shape, primal.stride(), dtype=dtype, device=primal.device).copy_(t)


def jvp(slices, modes, weights, positions, tangent_slices, tangent_modes, slice_thickness, voltage_kv, calib_ang,
        shift_calib_ang=None, batch: int = 0, windows=None, want_patterns: bool = True, lanes: int = 0):
    """(patterns or None, dI) for the tangent (tangent_slices, tangent_modes), either
    of which may be None (zero). Runs ``ptyro_ms_jvp``: the wave and its tangent go
    through the forward's passes together."""
    lib = _lib.load()
    dev = slices.device
    S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
    if not engine_grid(modes.shape[0], modes.shape[1]):
        return _jvp_any(lib, slices, modes, weights, positions, tangent_slices, tangent_modes, slice_thickness,
                        voltage_kv, calib_ang, calib_ang if shift_calib_ang is None else shift_calib_ang, batch,
                        windows, want_patterns)
    n, f = check_windows(slices, modes, windows, P)
    sc = float(calib_ang if shift_calib_ang is None else shift_calib_ang)
    ts = _like(tangent_slices, slices, torch.float32)
    tm = _like(tangent_modes, modes, torch.complex64)
    out = torch.empty((P, n, n), dtype=torch.float32, device=dev) if want_patterns else None
    tan = torch.empty((P, n, n), dtype=torch.float32, device=dev)
    if not P:
        return out, tan
    # contiguous probe ranges as concurrent tangent forwards on side streams (every
    # output is per probe, so the lanes change nothing but the overlap)
    if lanes == 0:
        lanes = 2 if P * n * n * M * 8 >= _LANE_MIN_WAVE_BYTES else 1
    lanes = max(1, min(int(lanes), P))
    main = torch.cuda.current_stream(dev)
    bounds = [P * i // lanes for i in range(lanes + 1)]
    streams = [main] if lanes == 1 else _side_streams(dev, lanes)
    # a slot holds the wave and its tangent: half the lane's share of the L2 wave budget
    lb = batch if (lanes == 1 or batch) else max(1, lane_batch(n, M, lanes) // 2)
    for (lo, hi), st in zip(zip(bounds[:-1], bounds[1:]), streams):
        win = None if windows is None else windows[lo:hi].contiguous()
        prm = ms_params(n, S, M, hi - lo, voltage_kv, slice_thickness, calib_ang, sc, slices.stride(), modes.stride(),
                        lb, 0, f, win)
        ws_bytes = lib.ptyro_ms_jvp_workspace_bytes(ctypes.byref(prm))
        ws = _workspace(ws_bytes, dev)
        if st is not main:
            st.wait_stream(main)
        with torch.cuda.stream(st):
            _lib.check(lib.ptyro_ms_jvp(ctypes.byref(prm), slices.data_ptr(), None if ts is None else ts.data_ptr(),
                                        modes.data_ptr(), None if tm is None else tm.data_ptr(), weights.data_ptr(),
                                        positions[lo:hi].data_ptr(), None if out is None else out[lo:hi].data_ptr(),
                                        tan[lo:hi].data_ptr(), ws.data_ptr(), ws_bytes, _stream_ptr(dev)))
        if st is not main:
            for t in (ws,) + (() if win is None else (win,)):
                t.record_stream(st)
    for st in streams:
        if st is not main:
            main.wait_stream(st)
    return out, tan


def _jvp_any(lib, slices, modes, weights, positions, tangent_slices, tangent_modes, slice_thickness, voltage_kv,
             calib_ang, shift_calib_ang, batch, windows, want_patterns):
    """``jvp`` on any height x width grid (ptyro_gm_jvp)."""
    dev = slices.device
    h, w = check_any_grid(slices, modes, windows)
    P = positions.shape[0]
    prm = any_grid_params(slices, modes, P, voltage_kv, slice_thickness, calib_ang, float(shift_calib_ang), batch)
    ts = _like(tangent_slices, slices, torch.float32)
    tm = _like(tangent_modes, modes, torch.complex64)
    out = torch.empty((P, h, w), dtype=torch.float32, device=dev) if want_patterns else None
    tan = torch.empty((P, h, w), dtype=torch.float32, device=dev)
    if P:
        ws_bytes = lib.ptyro_gm_jvp_workspace_bytes(ctypes.byref(prm), h, w)
        if ws_bytes == 0:
            _lib.check(_lib.PTYRO_ERR_INVALID)
        ws = _workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            _lib.check(lib.ptyro_gm_jvp(ctypes.byref(prm), h, w, slices.data_ptr(),
                                        None if ts is None else ts.data_ptr(), modes.data_ptr(),
                                        None if tm is None else tm.data_ptr(), weights.data_ptr(),
                                        positions.data_ptr(), None if out is None else out.data_ptr(), tan.data_ptr(),
                                        ws.data_ptr(), ws_bytes, _stream_ptr(dev)))
        _lib.check_workspace_status(ws, "jvp")
    return out, tan


def vjp(slices, modes, weights, positions, grad_patterns, slice_thickness, voltage_kv, calib_ang,
        shift_calib_ang=None, ckpt_every: int = DEFAULT_CKPT, batch: int = 0, windows=None, tune=None):
    """(patterns, dL/dV, dL/dmodes in JAX's convention) for dL/dpatterns = grad_patterns."""
    lib = _lib.load()
    dev = slices.device
    S, M, P = slices.shape[2], modes.shape[2], positions.shape[0]
    sc = float(calib_ang if shift_calib_ang is None else shift_calib_ang)
    if not engine_grid(modes.shape[0], modes.shape[1]):
        h, w = check_any_grid(slices, modes, windows)
        prm = any_grid_params(slices, modes, P, voltage_kv, slice_thickness, calib_ang, sc, batch)
        res = torch.empty(max(1, lib.ptyro_gm_residual_bytes(ctypes.byref(prm), h, w) // 4), dtype=torch.float32,
                          device=dev)
        status = _lib.new_status(dev)
        out = run_forward_any(slices, slice_thickness, modes, weights, positions, voltage_kv, calib_ang, sc,
                              batch=batch, status=status, residuals=res)
        _lib.check_status(status, "vjp forward")
        g_slices = torch.empty_strided(slices.shape, slices.stride(), dtype=torch.float32, device=dev)
        g_modes = torch.empty_strided(modes.shape, modes.stride(), dtype=torch.complex64, device=dev)
        if P == 0:
            g_slices.zero_()
            g_modes.zero_()
        else:
            Stem4dFunction._adjoint_any(lib, slices, modes, weights, positions, res, grad_patterns, slice_thickness,
                                        voltage_kv, calib_ang, sc, batch, g_slices, g_modes, None)
        return out, g_slices, g_modes
    n, f = check_windows(slices, modes, windows, P)
    k = _ckpt_for(S, ckpt_every, n, P * M)
    prm = ms_params(n, S, M, P, voltage_kv, slice_thickness, calib_ang, sc, slices.stride(), modes.stride(), batch,
                    default_tune(n) if tune is None else int(tune), f, windows)
    out = torch.empty((P, n, n), dtype=torch.float32, device=dev)
    res = torch.empty(max(1, lib.ptyro_ms_residual_bytes(ctypes.byref(prm), k) // 4), dtype=torch.float32,
                      device=dev)
    tn = prm.tune
    run_forward_ckpt(slices, modes, weights, positions, k, slice_thickness, voltage_kv, calib_ang, sc, batch, tn,
                     windows, out, res)
    g_slices = torch.empty_strided(slices.shape, slices.stride(), dtype=torch.float32, device=dev)
    g_modes = torch.empty_strided(modes.shape, modes.stride(), dtype=torch.complex64, device=dev)
    run_backward(slices, modes, weights, positions, res, grad_patterns, k, slice_thickness, voltage_kv, calib_ang, sc,
                 batch, tn, windows, g_slices, g_modes)
    return out, g_slices, g_modes


# ----------------------------------------------------------------------------- probe
class _Fft2Fn(torch.autograd.Function):
    """fft2 / ifft2 on the engine's kernels with their adjoints."""

    @staticmethod
    def forward(ctx, x, inverse: bool):
        from .simulations import fft2
        ctx.inverse = inverse
        return fft2(x, inverse=inverse)

    @staticmethod
    def backward(ctx, g):
        from .simulations import fft2
        n2 = g.shape[-1] * g.shape[-2]
        if ctx.inverse:  # y = F^H x / n2  ->  x_bar = F y_bar / n2
            return fft2(g, inverse=False) / n2, None
        return fft2(g, inverse=True) * n2, None  # y = F x -> x_bar = F^H y_bar


def make_probe_differentiable(voltage_kv: float, aperture_mrad: float, probe_shape, probe_calibration_pm: float,
                              defocus_ang, c3_ang, c5_ang=0.0, a1x_ang=0.0, a1y_ang=0.0,
                              device=None) -> torch.Tensor:
    """make_probe (multislice/simulations.py:334-431) with torch-differentiable
    aberration coefficients (tensors or floats).

    chi = 2 pi / lambda (C1 p^2/2 + 1e7 C3 p^4/4 + 1e7 C5 p^6/6) as the reference
    (:491-497), plus a two-fold astigmatism term (extension; the reference has
    none): 2 pi / lambda * p^2/2 * (A1x cos 2 phi + A1y sin 2 phi), phi the azimuth
    of q. The IFFT2 runs on the engine's kernels.
    """
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    h, w = int(probe_shape[0]), int(probe_shape[1])
    if not engine_grid(h, w) and not (1 <= h <= 4096 and 1 <= w <= 4096):
        raise ValueError(f"probe_shape must be in [1, 4096]^2, got ({h}, {w})")
    lam = relativistic_wavelength_ang(voltage_kv)

    def axis(m: int) -> torch.Tensor:
        # the reference's grid: arange(-m/2, m/2) rolled by m // 2, over the field of view
        a = torch.arange(m, dtype=torch.float64, device=dev) - m / 2.0
        return torch.roll(a, m // 2) / (m * 0.01 * float(probe_calibration_pm))
    ly, lx = torch.meshgrid(axis(h), axis(w), indexing="ij")
    q = torch.sqrt(lx * lx + ly * ly)
    mask = (q <= (aperture_mrad / 1000.0) / lam).to(torch.float64)
    p = lam * q

    def t(v):
        return v.to(torch.float64) if isinstance(v, torch.Tensor) else torch.tensor(float(v), dtype=torch.float64,
                                                                                     device=dev)
    chi = (t(defocus_ang) * p ** 2 / 2 + t(c3_ang) * 1e7 * p ** 4 / 4 + t(c5_ang) * 1e7 * p ** 6 / 6)
    phi = torch.atan2(ly, lx)
    chi = chi + p ** 2 / 2 * (t(a1x_ang) * torch.cos(2 * phi) + t(a1y_ang) * torch.sin(2 * phi))
    chi = 2 * math.pi * chi / lam
    a = torch.polar(mask, -chi).to(torch.complex64)
    probe = _Fft2Fn.apply(a, True)
    return torch.roll(probe, shifts=(-(h // 2), -(w // 2)), dims=(0, 1))  # ifftshift
