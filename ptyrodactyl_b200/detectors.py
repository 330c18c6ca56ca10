"""Virtual detectors: annular integration of 4D-STEM patterns, standalone or fused
into the forward model's pattern pass.

``annular_detector`` keeps the reference's signature and result
(multislice/simulations.py:1539-1656). ``stem_4d_annular`` and
``stem_4d_detectors`` run the forward with the integration done on each far-field
intensity while it is still in registers, so the (P, N, N) patterns never reach
HBM (P scalars per detector instead).

Masks follow the reference exactly: on the fftshifted grid, pixel (i, j) has
``q = sqrt((i - h//2)^2 + (j - w//2)^2) * fourier_calib`` and is inside an annulus
when ``inner/1000/lambda <= q <= outer/1000/lambda`` (simulations.py:1590-1618).
The host builds them in float64 and hands the kernels one uint32 per pixel in
UNSHIFTED frequency order, bit d for detector d.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .simulations import (
    _beam_on,
    _device,
    _stream_ptr,
    _workspace,
    check_windows,
    engine_grid,
    ms_params,
    relativistic_wavelength_ang,
)
from .types import (
    STEM4D,
    CalibratedArray,
    DetectorConfig,
    MicroscopeConfig,
    PotentialSlices,
    ProbeModes,
    as_tensor,
    create_calibrated_array,
)

Annulus = Tuple[float, float]


def annular_mask(shape, fourier_calib: float, voltage_kv: float, inner_mrad: float, outer_mrad: float) -> np.ndarray:
    """Boolean annulus on the fftshifted grid (simulations.py:1590-1618)."""
    wavelength = relativistic_wavelength_ang(voltage_kv)
    inner_k = (float(inner_mrad) / 1000.0) / wavelength
    outer_k = (float(outer_mrad) / 1000.0) / wavelength
    hh, ww = int(shape[0]), int(shape[1])
    qy = np.arange(hh) - hh // 2
    qx = np.arange(ww) - ww // 2
    qya, qxa = np.meshgrid(qy, qx, indexing="ij")
    q_radius = np.sqrt(qya ** 2 + qxa ** 2) * float(fourier_calib)
    return (q_radius >= inner_k) & (q_radius <= outer_k)


def detector_mask_bits(n: int, fourier_calib: float, voltage_kv: float, annuli: Sequence[Annulus],
                       device=None) -> torch.Tensor:
    """uint32 (n, n) per-pixel detector bits in unshifted frequency order, as an
    int32 CUDA tensor (same bits)."""
    if not 1 <= len(annuli) <= _lib.MAX_DETECTORS:
        raise ValueError(f"between 1 and {_lib.MAX_DETECTORS} detectors are supported, got {len(annuli)}")
    bits = np.zeros((n, n), dtype=np.uint32)
    for d, (inner, outer) in enumerate(annuli):
        if not (np.isfinite(inner) and np.isfinite(outer) and 0 <= inner <= outer):
            raise ValueError("annuli must satisfy 0 <= inner <= outer")
        bits |= annular_mask((n, n), fourier_calib, voltage_kv, inner, outer).astype(np.uint32) << np.uint32(d)
    unshifted = np.fft.ifftshift(bits)  # shifted pixel (i, j) holds frequency (i - n/2, j - n/2)
    return torch.from_numpy(unshifted.view(np.int32).copy()).to(_device(device))


def stored_mask_bits(shape, fourier_calib: float, voltage_kv: float, annuli: Sequence[Annulus],
                     device=None) -> torch.Tensor:
    """uint32 (h, w) per-pixel detector bits in the stored patterns' own
    (fftshifted) order, bit d for annulus d, as an int32 CUDA tensor (same bits):
    the reference's annular mask (simulations.py:1590-1618) at any height x width."""
    if not 1 <= len(annuli) <= _lib.MAX_DETECTORS:
        raise ValueError(f"between 1 and {_lib.MAX_DETECTORS} detectors are supported, got {len(annuli)}")
    hh, ww = int(shape[0]), int(shape[1])
    bits = np.zeros((hh, ww), dtype=np.uint32)
    for d, (inner, outer) in enumerate(annuli):
        if not (np.isfinite(inner) and np.isfinite(outer) and 0 <= inner <= outer):
            raise ValueError("annuli must satisfy 0 <= inner <= outer")
        bits |= annular_mask((hh, ww), fourier_calib, voltage_kv, inner, outer).astype(np.uint32) << np.uint32(d)
    return torch.from_numpy(bits.view(np.int32).copy()).to(_device(device))


def _annuli_of(detector: DetectorConfig, annuli: Optional[Sequence[Annulus]]) -> list:
    if annuli is None:
        return [(detector.collection_inner_mrad, detector.collection_outer_mrad)]
    return [(float(a), float(b)) for a, b in annuli]


def virtual_detectors(stem4d_data: STEM4D, annuli: Sequence[Annulus]) -> torch.Tensor:
    """(P, K) float64 masked sums of the stored (P, H, W) patterns, one column per
    annulus, at any pattern height x width."""
    data = stem4d_data.data
    if data.ndim != 3:
        raise ValueError("stem4d_data.data must be (P, H, W)")
    hh, ww = int(data.shape[1]), int(data.shape[2])
    if not (1 <= hh <= 8192 and 1 <= ww <= 8192):
        raise ValueError(f"pattern height and width must be in [1, 8192], got ({hh}, {ww})")
    dev = _device(data.device if data.is_cuda else None)
    pats = as_tensor(data, torch.float32, dev).contiguous()
    out = torch.empty((pats.shape[0], len(annuli)), dtype=torch.float64, device=dev)
    lib = _lib.load()
    if hh == ww and hh >= 2 and not hh & (hh - 1):
        mask = detector_mask_bits(hh, stem4d_data.fourier_space_calib, stem4d_data.voltage_kv, annuli, dev)
        rc = lib.ptyro_detect_patterns(pats.data_ptr(), pats.shape[0], hh, mask.data_ptr(), len(annuli),
                                       out.data_ptr(), _stream_ptr(dev))
    else:
        mask = stored_mask_bits((hh, ww), stem4d_data.fourier_space_calib, stem4d_data.voltage_kv, annuli, dev)
        rc = lib.ptyro_detect_patterns_hw(pats.data_ptr(), pats.shape[0], hh, ww, mask.data_ptr(), len(annuli),
                                          out.data_ptr(), _stream_ptr(dev))
    _lib.check(rc)
    return out


def _image(values: torch.Tensor, detector: DetectorConfig, calib: float) -> CalibratedArray:
    ny, nx = detector.scan_shape
    return create_calibrated_array(values.reshape(ny, nx), calib, calib, True)


def annular_detector(stem4d_data: STEM4D, detector: DetectorConfig) -> CalibratedArray:
    """Integrate 4D-STEM data with an annular detector (simulations.py:1539-1656):
    float64 image (ny, nx) with the real-space calibration of ``stem4d_data``."""
    if detector.scan_shape is None:
        raise ValueError("detector.scan_shape is required")
    vals = virtual_detectors(stem4d_data, _annuli_of(detector, None))
    return _image(vals[:, 0], detector, stem4d_data.real_space_calib)


def run_forward_detect(slices: torch.Tensor, slice_thickness: float, modes: torch.Tensor, weights: torch.Tensor,
                       positions: torch.Tensor, voltage_kv: float, calib_ang: float, shift_calib_ang: float,
                       mask: torch.Tensor, num_det: int, out: Optional[torch.Tensor] = None,
                       patterns: Optional[torch.Tensor] = None, accumulate: bool = False, tune: int = 0,
                       batch: int = 0) -> torch.Tensor:
    """Device-level fused forward + detectors: returns (P, num_det) float64; also
    fills ``patterns`` (P, n, n) float32 when given."""
    lib = _lib.load()
    dev = slices.device
    num_probes = positions.shape[0]
    n, f = check_windows(slices, modes, None, num_probes)
    prm = ms_params(n, slices.shape[2], modes.shape[2], num_probes, voltage_kv, slice_thickness, calib_ang,
                    shift_calib_ang, slices.stride(), modes.stride(), batch, tune, f, None,
                    _lib.PTYRO_FLAG_ACCUMULATE if accumulate else 0)
    if out is None:
        out = (torch.zeros if accumulate else torch.empty)((num_probes, num_det), dtype=torch.float64, device=dev)
    if num_probes == 0:
        return out
    ws_bytes = lib.ptyro_ms_detect_workspace_bytes(ctypes.byref(prm), num_det)
    if ws_bytes == 0:
        _lib.check(_lib.PTYRO_ERR_INVALID)
    ws = _workspace(ws_bytes, dev)
    rc = lib.ptyro_ms_forward_detect(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(), weights.data_ptr(),
                                     positions.data_ptr(), mask.data_ptr(), num_det, out.data_ptr(),
                                     None if patterns is None else patterns.data_ptr(), ws.data_ptr(), ws_bytes,
                                     _stream_ptr(dev))
    _lib.check(rc)
    return out


def stem_4d_detectors(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
                      detector: DetectorConfig, annuli: Optional[Sequence[Annulus]] = None) -> torch.Tensor:
    """``virtual_detectors(stem_4d(...), annuli)`` in one fused forward: (P, K)
    float64, no pattern stored. ``annuli`` defaults to the detector's own
    (collection_inner_mrad, collection_outer_mrad). With ensemble axes, or on a grid
    other than the pass engine's square power-of-two edges, the integration runs on
    stem_4d's patterns instead, 1024 probes at a time (same values)."""
    if detector.scan_positions_px is None:
        raise ValueError("detector.scan_positions_px is required")
    dev = _device(pot_slice.slices.device if pot_slice.slices.is_cuda else None)
    slices = as_tensor(pot_slice.slices, torch.float32, dev)
    if slices.ndim == 2:
        slices = slices[..., None]
    modes, weights = _beam_on(beam, dev)
    n = modes.shape[0]
    if not microscope.ensemble.is_empty() or not engine_grid(modes.shape[0], modes.shape[1]):
        # ensemble axes and any-size grids: stem_4d's own path, then the masked sums
        # of its patterns, a chunk of probes at a time
        return _detectors_unfused(pot_slice, beam, microscope, detector, _annuli_of(detector, annuli))
    positions = as_tensor(detector.scan_positions_px, torch.float64, dev).reshape(-1, 2).contiguous()
    calib = min(float(pot_slice.calib), float(beam.calib))
    rings = _annuli_of(detector, annuli)
    mask = detector_mask_bits(n, 1.0 / (n * calib), microscope.voltage_kv, rings, dev)
    return run_forward_detect(slices, pot_slice.slice_thickness, modes, weights, positions, microscope.voltage_kv,
                              calib, detector.real_space_calib_ang, mask, len(rings))


def _detectors_unfused(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
                       detector: DetectorConfig, rings: list, chunk: int = 1024) -> torch.Tensor:
    from .simulations import stem_4d
    from .types import create_detector_config
    pos = detector.scan_positions_px
    parts = []
    for c0 in range(0, pos.shape[0], int(chunk)):
        sub = create_detector_config(detector.real_space_calib_ang, detector.probe_calibration_pm,
                                     detector.collection_inner_mrad, detector.collection_outer_mrad,
                                     scan_positions_px=pos[c0:c0 + int(chunk)])
        parts.append(virtual_detectors(stem_4d(pot_slice, beam, microscope, sub), rings))
    return torch.cat(parts, dim=0)


def stem_4d_annular(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
                    detector: DetectorConfig) -> CalibratedArray:
    """``annular_detector(stem_4d(pot_slice, beam, microscope, detector), detector)``
    with the integration fused into the forward's pattern pass."""
    if detector.scan_shape is None:
        raise ValueError("detector.scan_shape is required")
    vals = stem_4d_detectors(pot_slice, beam, microscope, detector)
    return _image(vals[:, 0], detector, detector.real_space_calib_ang)


# ----------------------------------------------------------------------------- CBED clip + resize
def linear_resize_weights(input_size: int, output_size: int, antialias: bool = True) -> np.ndarray:
    """(output_size, input_size) weights of a linear (triangle-kernel) resize with
    half-pixel centres, widened by the downscale factor when antialiasing, each
    output row normalised to unit sum and zero where the sample falls outside the
    input: the scale-and-translate weights of jax.image.resize(method="linear")
    (jax 0.9.2, jax/_src/image/scale.py), restated."""
    scale = output_size / input_size
    inv_scale = 1.0 / scale
    kernel_scale = max(inv_scale, 1.0) if antialias else 1.0
    sample_f = (np.arange(output_size) + 0.5) * inv_scale - 0.5
    x = np.abs(sample_f[None, :] - np.arange(input_size, dtype=np.float64)[:, None]) / kernel_scale
    weights = np.maximum(0.0, 1.0 - x)
    total = np.sum(weights, axis=0, keepdims=True)
    weights = np.where(np.abs(total) > 1000.0 * float(np.finfo(np.float32).eps),
                       weights / np.where(total != 0, total, 1), 0.0)
    inside = (sample_f >= -0.5) & (sample_f <= input_size - 0.5)
    return np.where(inside[None, :], weights, 0.0).T


def _crop_bounds(h: int, w: int, fourier_calib_inv_ang: float, voltage_kv: float, extent_mrad: float) -> tuple:
    mrad_per_inv_ang = relativistic_wavelength_ang(voltage_kv) * 1000.0
    extent_pixels = int(np.ceil((float(extent_mrad) / mrad_per_inv_ang) / float(fourier_calib_inv_ang)))
    cy, cx = h // 2, w // 2
    y0, y1 = max(0, cy - extent_pixels), min(h, cy + extent_pixels)
    x0, x1 = max(0, cx - extent_pixels), min(w, cx + extent_pixels)
    return y0, y1, x0, x1


def clip_cbed(cbed: torch.Tensor, fourier_calib_inv_ang: float, voltage_kv: float, extent_mrad: float,
              output_shape: Tuple[int, int]) -> torch.Tensor:
    """Central crop of ``extent_mrad`` (half angle) and linear resize to
    ``output_shape`` (plots/figuring.py:37-117) of one (H, W) pattern or a (P, H, W)
    stack, float32 on the device."""
    dev = _device(cbed.device if cbed.is_cuda else None)
    pats = as_tensor(cbed, torch.float32, dev)
    single = pats.ndim == 2
    if single:
        pats = pats[None]
    if pats.ndim != 3:
        raise ValueError("cbed must be (H, W) or (P, H, W)")
    pats = pats.contiguous()
    p, h, w = pats.shape
    ho, wo = (int(v) for v in output_shape)
    y0, y1, x0, x1 = _crop_bounds(h, w, fourier_calib_inv_ang, voltage_kv, extent_mrad)
    hc, wc = y1 - y0, x1 - x0
    if hc <= 0 or wc <= 0:
        raise ValueError("extent_mrad selects no pixels")
    wy = linear_resize_weights(hc, ho) if ho != hc else np.eye(hc)
    wx = linear_resize_weights(wc, wo) if wo != wc else np.eye(wc)
    wy_d = torch.as_tensor(wy.astype(np.float32), device=dev).contiguous()
    wx_d = torch.as_tensor(wx.astype(np.float32), device=dev).contiguous()
    out = torch.empty((p, ho, wo), dtype=torch.float32, device=dev)
    lib = _lib.load()
    nbytes = lib.ptyro_clip_resize_workspace_bytes(p, hc, wo)
    ws = _workspace(nbytes, dev)
    _lib.check(lib.ptyro_clip_resize(pats.data_ptr(), p, h, w, y0, x0, hc, wc, wy_d.data_ptr(), ho, wx_d.data_ptr(),
                                     wo, out.data_ptr(), ws.data_ptr(), nbytes, _stream_ptr(dev)))
    return out[0] if single else out


def stem_4d_clipped(pot_slice: PotentialSlices, beam: ProbeModes, microscope: MicroscopeConfig,
                    detector: DetectorConfig, cbed_extent_mrad: float, cbed_shape: Tuple[int, int],
                    chunk: int = 1024) -> STEM4D:
    """4D-STEM with every pattern clipped to ``cbed_extent_mrad`` and resized to
    ``cbed_shape``, as the reference's 4D-STEM workflow stores them
    (workflows/stem_4d.py:488-540): the forward runs ``chunk`` probes at a time so the
    full-size patterns of only one chunk exist in device memory. The output Fourier
    calibration is ``2 extent / cbed_shape[0]`` mrad per pixel, in 1/Angstrom."""
    from .simulations import stem_4d
    from .types import create_detector_config, create_stem4d
    if detector.scan_positions_px is None:
        raise ValueError("detector.scan_positions_px is required")
    pos = detector.scan_positions_px
    parts = []
    s4 = None
    for c0 in range(0, pos.shape[0], int(chunk)):
        sub = create_detector_config(detector.real_space_calib_ang, detector.probe_calibration_pm,
                                     detector.collection_inner_mrad, detector.collection_outer_mrad,
                                     scan_positions_px=pos[c0:c0 + int(chunk)])
        s4 = stem_4d(pot_slice, beam, microscope, sub)
        parts.append(clip_cbed(s4.data, s4.fourier_space_calib, microscope.voltage_kv, cbed_extent_mrad, cbed_shape))
    data = torch.cat(parts, dim=0)
    mrad_per_inv_ang = relativistic_wavelength_ang(microscope.voltage_kv) * 1000.0
    fourier = (2.0 * float(cbed_extent_mrad) / int(cbed_shape[0])) / mrad_per_inv_ang
    return create_stem4d(data, detector.real_space_calib_ang, fourier,
                         pos.to(torch.float64) * detector.real_space_calib_ang, microscope.voltage_kv)
