"""Oracle (test infrastructure only): NumPy restatement of ptyrodactyl's multislice path.

This module is the CPU checker for the CUDA kernels in ``ptyrodactyl_b200``. It
is never called by the product path: only ``tests/``, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` import it.

Every function follows the reference's arithmetic in operation order. Paths
are relative to the reference project root. ``dtype`` selects the wave
precision: ``np.complex128`` restates the reference as shipped (the package
forces x64, ``src/ptyrodactyl/__init__.py:96``); ``np.complex64`` restates its
float32 path (wave, propagator and transmission held in complex64; physics
scalars evaluated in float64 and rounded where they enter an array).

Pinned against the reference's golden file
``tests/test_data/plan01_ug_reference.npz`` (see ``tests/golden/make_golden.py``
and ``tests/test_oracle.py``).
"""

from __future__ import annotations

import numpy as np

# CODATA 2018 exact/recommended values, types/constants.py:60-96
H_PLANCK = 6.62607015e-34
M_E = 9.1093837015e-31
E_CHARGE = 1.602176634e-19
C_LIGHT = 2.99792458e8


def relativistic_wavelength_ang(voltage_kv: float) -> float:
    """lambda = h c / sqrt(eV (2 m c^2 + eV)) in Angstrom (types/constants.py:291-340)."""
    ev = float(voltage_kv) * 1000.0 * E_CHARGE
    numerator = (H_PLANCK * H_PLANCK) * (C_LIGHT * C_LIGHT)
    denominator = ev * (2.0 * M_E * (C_LIGHT * C_LIGHT) + ev)
    return 1e10 * np.sqrt(numerator / denominator)


def interaction_sigma(voltage_kv: float) -> float:
    """sigma = 2 pi / (lambda V) (m c^2 + eV) / (2 m c^2 + eV) (multislice/simulations.py:150-157)."""
    voltage = float(voltage_kv) * 1000.0
    ev = E_CHARGE * voltage
    lam = relativistic_wavelength_ang(voltage_kv)
    einstein = M_E * (C_LIGHT * C_LIGHT)
    return ((2 * np.pi / (lam * voltage)) * (einstein + ev)) / ((2 * einstein) + ev)


def transmission_func(pot_slice: np.ndarray, voltage_kv: float, dtype=np.complex128) -> np.ndarray:
    """T = exp(i sigma V) (multislice/simulations.py:105-159)."""
    sigma = interaction_sigma(voltage_kv)
    return np.exp(1j * sigma * np.asarray(pot_slice, dtype=np.float64)).astype(dtype)


def propagation_func(h: int, w: int, thickness_ang: float, voltage_kv: float, calib_ang: float,
                     dtype=np.complex128) -> np.ndarray:
    """P(q) = exp(-i pi lambda dz |q|^2), q = fftfreq(n, d=calib) (multislice/simulations.py:162-225)."""
    qy = np.fft.fftfreq(int(h), d=float(calib_ang))
    qx = np.fft.fftfreq(int(w), d=float(calib_ang))
    lya, lxa = np.meshgrid(qy, qx, indexing="ij")
    l_sq = np.square(lxa) + np.square(lya)
    lam = relativistic_wavelength_ang(voltage_kv)
    prop = np.exp((-1j) * np.pi * lam * float(thickness_ang) * l_sq)
    return prop.astype(dtype)


def aberration(fourier_coord: np.ndarray, lambda_angstrom: float, defocus: float = 0.0,
               c3: float = 0.0, c5: float = 0.0) -> np.ndarray:
    """chi = 2 pi / lambda (C1 p^2/2 + 1e7 C3 p^4/4 + 1e7 C5 p^6/6), p = lambda q
    (multislice/simulations.py:434-498). The 1e7 factor makes the C3/C5 fields act as mm."""
    p = lambda_angstrom * fourier_coord
    chi = ((defocus * np.power(p, 2)) / 2) + ((c3 * 1e7 * np.power(p, 4)) / 4) + \
        ((c5 * 1e7 * np.power(p, 6)) / 6)
    return (2 * np.pi * chi) / lambda_angstrom


def probe_fourier_radius(probe_shape, probe_calibration_pm: float) -> np.ndarray:
    """|q| on the unshifted grid that make_probe builds (multislice/simulations.py:400-416)."""
    image_y, image_x = int(probe_shape[0]), int(probe_shape[1])
    x_fov = image_x * 0.01 * float(probe_calibration_pm)
    y_fov = image_y * 0.01 * float(probe_calibration_pm)
    qx = np.arange(-image_x / 2, image_x / 2, 1) / x_fov
    qy = np.arange(-image_y / 2, image_y / 2, 1) / y_fov
    lx = np.roll(qx, image_x // 2)
    ly = np.roll(qy, image_y // 2)
    lya, lxa = np.meshgrid(lx, ly)  # 'xy' indexing, as the reference
    l2 = np.multiply(lxa, lxa) + np.multiply(lya, lya)
    return l2 ** 0.5


def make_probe(voltage_kv: float, aperture_mrad: float, probe_shape, probe_calibration_pm: float,
               defocus_ang: float = 0.0, c3_ang: float = 0.0, c5_ang: float = 0.0,
               dtype=np.complex128) -> np.ndarray:
    """Aperture mask |q| <= alpha/lambda times exp(-i chi), then ifftshift(ifft2(.))
    (multislice/simulations.py:334-431). The result is unnormalised:
    sum |psi|^2 = n_aperture / (H W)."""
    aperture = aperture_mrad / 1000.0
    wavelength = relativistic_wavelength_ang(voltage_kv)
    l_max = aperture / wavelength
    q = probe_fourier_radius(probe_shape, probe_calibration_pm)
    a_dist = np.asarray(q <= l_max, dtype=np.complex128)
    chi = aberration(q, wavelength, defocus_ang, c3_ang, c5_ang)
    a_dist = a_dist * np.exp(-1j * chi)
    return np.fft.ifftshift(np.fft.ifft2(a_dist)).astype(dtype)


def shift_beam_fourier(beam: np.ndarray, pos: np.ndarray, calib_ang: float,
                       dtype=np.complex128) -> np.ndarray:
    """psi_p = ifft2(fft2(psi) exp(-2 pi i (qy y_p + qx x_p))), q in 1/Angstrom, pos in
    Angstrom (multislice/simulations.py:1236-1327). (H,W,M) + (P,2) -> (P,H,W,M)."""
    our_beam = np.asarray(beam).astype(dtype)
    if our_beam.ndim == 2:
        our_beam = our_beam[..., None]
    hh, ww = our_beam.shape[0], our_beam.shape[1]
    pos = np.atleast_2d(np.asarray(pos, dtype=np.float64))
    qy = np.fft.fftfreq(hh, d=float(calib_ang))
    qx = np.fft.fftfreq(ww, d=float(calib_ang))
    qya, qxa = np.meshgrid(qy, qx, indexing="ij")
    beam_k = np.fft.fft2(our_beam, axes=(0, 1))
    out = np.empty((pos.shape[0], hh, ww, our_beam.shape[2]), dtype=dtype)
    for i in range(pos.shape[0]):
        phase = -2.0 * np.pi * ((qya * pos[i, 0]) + (qxa * pos[i, 1]))
        ramp = np.exp(1j * phase).astype(dtype)
        out[i] = np.fft.ifft2(beam_k * ramp[..., None], axes=(0, 1))
    return out


def cbed_amplitude(slices: np.ndarray, slice_thickness: float, voltage_kv: float,
                   calib_ang: float, beam_modes: np.ndarray, dtype=np.complex128) -> np.ndarray:
    """The slice loop (multislice/simulations.py:501-603): per slice wave *= T_s, then,
    unless it is the last slice, wave = ifft2(fft2(wave) * P); finally
    fftshift(fft2(wave)). slices (H,W,S), beam_modes (H,W,M) -> (H,W,M)."""
    slices = np.atleast_3d(np.asarray(slices, dtype=np.float64))
    wave = np.atleast_3d(np.asarray(beam_modes)).astype(dtype)
    h, w, num_slices = slices.shape
    prop = propagation_func(wave.shape[0], wave.shape[1], slice_thickness, voltage_kv,
                            calib_ang, dtype)
    for s in range(num_slices):
        trans = transmission_func(slices[:, :, s], voltage_kv, dtype)
        wave = wave * trans[..., None]
        if s != num_slices - 1:
            w_k = np.fft.fft2(wave, axes=(0, 1)) * prop[..., None]
            wave = np.fft.ifft2(w_k, axes=(0, 1)).astype(dtype)
    return np.fft.fftshift(np.fft.fft2(wave, axes=(0, 1)), axes=(0, 1))


def incoherent_intensity(amplitudes: np.ndarray, weights: np.ndarray) -> np.ndarray:
    """I = sum_m w_m |A_m|^2 (multislice/reduce.py:81-86); amplitudes (H,W,M)."""
    return np.einsum("n,hwn->hw", np.asarray(weights, np.float64), np.abs(amplitudes) ** 2)


def normalized_weights(weights) -> np.ndarray:
    """Weights divided by their sum (types/electron_types.py:1318-1324)."""
    w = np.asarray(weights, dtype=np.float64)
    return w / np.sum(w)


def cbed_image(slices, slice_thickness, pot_calib, beam_modes, weights, beam_calib,
               voltage_kv, dtype=np.complex128) -> np.ndarray:
    """Plain (no-ensemble) branch of cbed_image (multislice/simulations.py:1195-1233)."""
    calib = min(float(pot_calib), float(beam_calib))
    amps = cbed_amplitude(slices, slice_thickness, voltage_kv, calib, beam_modes, dtype)
    return incoherent_intensity(amps, weights)


def stem_4d(slices, slice_thickness, pot_calib, beam_modes, weights, beam_calib, voltage_kv,
            scan_positions_px, real_space_calib_ang, dtype=np.complex128) -> dict:
    """stem_4d (multislice/simulations.py:1330-1443).

    ``scan_positions_px`` is passed unchanged to ``shift_beam_fourier`` whose q is in
    1/Angstrom, so each position acts as Angstrom relative to the probe's own place
    (periodic); the output ``scan_positions`` claims ``pos * calib`` Angstrom.
    Returns a dict with the STEM4D fields; ``data`` is (P,H,W) float64.
    """
    positions = np.atleast_2d(np.asarray(scan_positions_px, dtype=np.float64))
    shifted = shift_beam_fourier(beam_modes, positions, real_space_calib_ang, dtype)
    calib = min(float(pot_calib), float(beam_calib))
    data = np.empty((positions.shape[0], shifted.shape[1], shifted.shape[2]), np.float64)
    for i in range(positions.shape[0]):
        amps = cbed_amplitude(slices, slice_thickness, voltage_kv, calib, shifted[i], dtype)
        data[i] = incoherent_intensity(amps, weights)
    return {
        "data": data,
        "real_space_calib": float(real_space_calib_ang),
        "fourier_space_calib": 1.0 / (shifted.shape[1] * calib),
        "scan_positions": positions * float(real_space_calib_ang),
        "voltage_kv": float(voltage_kv),
    }


# ---------------------------------------------------------------------------
# Adjoint (hand-derived), the checker for the gradient kernels.
#
# Forward per probe p and mode m:  phi_s = psi_s * T_s,  psi_{s+1} = U phi_s
# (U = ifft2 diag(P) fft2, unitary), A = fftshift(fft2(phi_{S-1})), I = sum_m w_m |A_m|^2.
# With g = dL/dI (real) and lam = dL/dconj(.) :
#   lam_A   = w_m g A
#   lam_phi = N^2 ifft2(ifftshift(lam_A))          (adjoint of fftshift o fft2)
#   dL/dV_s = 2 sigma Im(conj(phi_s) lam_phi_s)     (T = exp(i sigma V))
#   lam_psi = conj(T_s) lam_phi ;  lam_phi_{s-1} = U^H lam_psi = ifft2(conj(P) fft2(lam_psi))
#   lam_beam = sum_p N^2 ifft2? -> via shift adjoint below.
# JAX's gradient of a real loss w.r.t. a complex input z is 2 dL/dz = conj(2 lam_z).
# ---------------------------------------------------------------------------


def stem_4d_vjp(slices, slice_thickness, pot_calib, beam_modes, weights, beam_calib, voltage_kv,
                scan_positions_px, real_space_calib_ang, g, dtype=np.complex128, with_positions=False):
    """Gradient of L with dL/d data = g (P,H,W) through stem_4d.

    Returns (dV (H,W,S) float64, dbeam (H,W,M) complex in JAX's convention
    conj(2 dL/dconj(beam))), and with ``with_positions`` also dL/d(positions) (P, 2):
    psi0_p = ifft2(fft2(beam) R_p) and dL/dy_p = 2 Re sum conj(lam_psi0) d psi0/dy_p.
    Weights are treated as constants.
    """
    slices = np.atleast_3d(np.asarray(slices, dtype=np.float64))
    h, w, num_slices = slices.shape
    positions = np.atleast_2d(np.asarray(scan_positions_px, dtype=np.float64))
    beam = np.atleast_3d(np.asarray(beam_modes)).astype(dtype)
    n_modes = beam.shape[2]
    weights = np.asarray(weights, np.float64)
    calib = min(float(pot_calib), float(beam_calib))
    sigma = interaction_sigma(voltage_kv)
    prop = propagation_func(h, w, slice_thickness, voltage_kv, calib, dtype)
    trans = [transmission_func(slices[:, :, s], voltage_kv, dtype) for s in range(num_slices)]
    shifted = shift_beam_fourier(beam, positions, real_space_calib_ang, dtype)
    dv = np.zeros((h, w, num_slices), np.float64)
    # adjoint of the shift: psi_p = ifft2(fft2(beam) ramp_p)
    qy = np.fft.fftfreq(h, d=float(real_space_calib_ang))
    qx = np.fft.fftfreq(w, d=float(real_space_calib_ang))
    qya, qxa = np.meshgrid(qy, qx, indexing="ij")
    lam_beam_k = np.zeros((h, w, n_modes), np.complex128)
    dpos = np.zeros((positions.shape[0], 2))
    beam_k = np.fft.fft2(beam, axes=(0, 1))
    for i in range(positions.shape[0]):
        phis = []
        wave = shifted[i].copy()
        for s in range(num_slices):
            phi = wave * trans[s][..., None]
            phis.append(phi)
            if s != num_slices - 1:
                wave = np.fft.ifft2(np.fft.fft2(phi, axes=(0, 1)) * prop[..., None],
                                    axes=(0, 1)).astype(dtype)
        amp = np.fft.fftshift(np.fft.fft2(phis[-1], axes=(0, 1)), axes=(0, 1))
        lam_a = weights[None, None, :] * g[i][..., None] * amp
        lam = (h * w) * np.fft.ifft2(np.fft.ifftshift(lam_a, axes=(0, 1)), axes=(0, 1))
        for s in range(num_slices - 1, -1, -1):
            dv[:, :, s] += 2.0 * sigma * np.sum(np.imag(np.conj(phis[s]) * lam), axis=2)
            lam = np.conj(trans[s])[..., None] * lam
            if s > 0:
                lam = np.fft.ifft2(np.conj(prop)[..., None] * np.fft.fft2(lam, axes=(0, 1)),
                                   axes=(0, 1))
        # psi = ifft2(B ramp) -> lam_B = conj(ramp) * fft2(lam)/(HW)
        phase = -2.0 * np.pi * ((qya * positions[i, 0]) + (qxa * positions[i, 1]))
        ramp = np.exp(1j * phase)
        if with_positions:
            for c, q in enumerate((qya, qxa)):
                dpsi = np.fft.ifft2(beam_k * (ramp * (-2j * np.pi * q))[..., None], axes=(0, 1))
                dpos[i, c] = 2.0 * np.real(np.sum(np.conj(lam) * dpsi))
        lam_beam_k += np.conj(ramp)[..., None] * np.fft.fft2(lam, axes=(0, 1)) / (h * w)
    # B = fft2(beam) -> lam_beam = (HW) ifft2(lam_B)
    lam_beam = (h * w) * np.fft.ifft2(lam_beam_k, axes=(0, 1))
    if with_positions:
        return dv, np.conj(2.0 * lam_beam), dpos
    return dv, np.conj(2.0 * lam_beam)


def aperture_count(voltage_kv, aperture_mrad, probe_shape, probe_calibration_pm) -> int:
    """Number of pixels inside the hard aperture; sum of every stem_4d pattern."""
    lam = relativistic_wavelength_ang(voltage_kv)
    q = probe_fourier_radius(probe_shape, probe_calibration_pm)
    return int(np.count_nonzero(q <= (aperture_mrad / 1000.0) / lam))


def stem_4d_windowed(field, slice_thickness, pot_calib, beam_modes, weights, beam_calib, voltage_kv,
                     scan_positions_px, real_space_calib_ang, windows, dtype=np.complex128):
    """Probe p sees the n x n window of the periodic field (F, F, S) starting at
    windows[p]; otherwise stem_4d. (The reference crops a tile per position in
    workflows/stem_4d.py:553; here the crop is periodic.)"""
    n = np.atleast_3d(beam_modes).shape[0]
    pos = np.atleast_2d(np.asarray(scan_positions_px, np.float64))
    out = np.empty((pos.shape[0], n, n), np.float64)
    for i, (wy, wx) in enumerate(np.asarray(windows)):
        win = np.roll(field, (-int(wy), -int(wx)), axis=(0, 1))[:n, :n]
        out[i] = stem_4d(win, slice_thickness, pot_calib, beam_modes, weights, beam_calib, voltage_kv, pos[i:i + 1],
                         real_space_calib_ang, dtype)["data"][0]
    return out


def stem_4d_windowed_vjp(field, slice_thickness, pot_calib, beam_modes, weights, beam_calib, voltage_kv,
                         scan_positions_px, real_space_calib_ang, windows, g, dtype=np.complex128):
    """(dL/dfield, dL/dbeam JAX convention) of stem_4d_windowed for dL/ddata = g."""
    beam = np.atleast_3d(beam_modes)
    n = beam.shape[0]
    pos = np.atleast_2d(np.asarray(scan_positions_px, np.float64))
    dfield = np.zeros(field.shape, np.float64)
    dbeam = np.zeros(beam.shape, np.complex128)
    for i, (wy, wx) in enumerate(np.asarray(windows)):
        rolled = np.roll(field, (-int(wy), -int(wx)), axis=(0, 1))
        dv, db = stem_4d_vjp(rolled[:n, :n], slice_thickness, pot_calib, beam, weights, beam_calib, voltage_kv,
                             pos[i:i + 1], real_space_calib_ang, g[i:i + 1], dtype)
        acc = np.zeros(field.shape, np.float64)
        acc[:n, :n] = dv
        dfield += np.roll(acc, (int(wy), int(wx)), axis=(0, 1))
        dbeam += db
    return dfield, dbeam


def slice_potential_from_atoms(atom_coords, atom_types, z_min, z_max, atom_potentials, grid_shape, calib_ang,
                               atom_mask=None) -> np.ndarray:
    """_compute_slice_potential (multislice/parallelized.py:54-169): atoms with
    z_min <= z < z_max scattered to floor(coord / calib) mod grid per type, each type's
    delta grid circularly convolved with its kernel by FFT, summed over types."""
    h, w = int(grid_shape[0]), int(grid_shape[1])
    coords = np.asarray(atom_coords, np.float64)
    types = np.asarray(atom_types)
    in_slice = ((coords[:, 2] >= z_min) & (coords[:, 2] < z_max)).astype(np.float64)
    if atom_mask is not None:
        in_slice = in_slice * np.asarray(atom_mask, np.float64)
    x_idx = np.mod(np.floor(coords[:, 0] / calib_ang).astype(np.int64), w)
    y_idx = np.mod(np.floor(coords[:, 1] / calib_ang).astype(np.int64), h)
    out = np.zeros((h, w), np.float64)
    pots = np.asarray(atom_potentials, np.float64)
    for t in range(pots.shape[0]):
        grid = np.zeros((h, w), np.float64)
        np.add.at(grid, (y_idx, x_idx), (types == t) * in_slice)
        out += np.real(np.fft.ifft2(np.fft.fft2(grid) * np.fft.fft2(pots[t])))
    return out


def stem4d_sharded(beam_modes, weights, atom_coords, atom_types, slice_z_bounds, atom_potentials, voltage_kv,
                   real_space_calib_ang, scan_positions_ang, atom_mask=None, dtype=np.complex128) -> dict:
    """stem4d_sharded (multislice/parallelized.py:348-536) without a mesh: slices built
    from atoms (thickness = first slice's z extent), positions in Angstrom, every
    calibration = detector.real_space_calib_ang."""
    beam = np.atleast_3d(np.asarray(beam_modes))
    h, w = beam.shape[0], beam.shape[1]
    bounds = np.asarray(slice_z_bounds, np.float64)
    slices = np.stack([slice_potential_from_atoms(atom_coords, atom_types, b[0], b[1], atom_potentials, (h, w),
                                                  real_space_calib_ang, atom_mask) for b in bounds], axis=-1)
    thickness = bounds[0, 1] - bounds[0, 0]
    out = stem_4d(slices, thickness, real_space_calib_ang, beam, weights, real_space_calib_ang, voltage_kv,
                  scan_positions_ang, real_space_calib_ang, dtype)
    out["scan_positions"] = np.atleast_2d(np.asarray(scan_positions_ang, np.float64))
    out["slices"] = slices
    return out


def annular_mask(shape, fourier_calib, voltage_kv, inner_mrad, outer_mrad):
    """Annulus on the fftshifted grid (simulations.py:1590-1618)."""
    wavelength = relativistic_wavelength_ang(voltage_kv)
    inner_k = (inner_mrad / 1000.0) / wavelength
    outer_k = (outer_mrad / 1000.0) / wavelength
    hh, ww = shape
    qya, qxa = np.meshgrid(np.arange(hh) - hh // 2, np.arange(ww) - ww // 2, indexing="ij")
    q_radius = np.sqrt(qya ** 2 + qxa ** 2) * fourier_calib
    return (q_radius >= inner_k) & (q_radius <= outer_k)


def annular_detector(data, fourier_calib, voltage_kv, inner_mrad, outer_mrad, scan_shape):
    """simulations.py:1539-1656: sum of each (fftshifted) pattern inside the
    annulus, reshaped to the scan raster."""
    data = np.asarray(data, dtype=np.float64)
    mask = annular_mask(data.shape[1:], fourier_calib, voltage_kv, inner_mrad, outer_mrad)
    return np.sum(data * mask, axis=(1, 2)).reshape(scan_shape)


# ---------------------------------------------------------------------------
# Tangent (forward-mode) restatement, the checker for the JVP kernels: what
# jax.jvp computes through stem_4d (jacobian/operators.py:30-80 takes it).
#   dpsi_0 = shift(dbeam);  dphi_s = T_s (dpsi_s + i sigma dV_s psi_s)
#   dpsi_{s+1} = U dphi_s;  dI = sum_m w_m 2 Re(conj(A_m) dA_m)
# ---------------------------------------------------------------------------


def stem_4d_jvp(slices, slice_thickness, pot_calib, beam_modes, weights, beam_calib, voltage_kv,
                scan_positions_px, real_space_calib_ang, dslices=None, dbeam=None, dtype=np.complex128):
    """(data, ddata): patterns and their directional derivative along
    (dslices, dbeam) (either may be None = zero); shapes as stem_4d's."""
    slices = np.atleast_3d(np.asarray(slices, dtype=np.float64))
    beam = np.atleast_3d(np.asarray(beam_modes)).astype(dtype)
    dsl = np.zeros_like(slices) if dslices is None else np.atleast_3d(np.asarray(dslices, dtype=np.float64))
    db = np.zeros_like(beam) if dbeam is None else np.atleast_3d(np.asarray(dbeam)).astype(dtype)
    positions = np.atleast_2d(np.asarray(scan_positions_px, dtype=np.float64))
    w = np.asarray(weights, np.float64)
    calib = min(float(pot_calib), float(beam_calib))
    sigma = interaction_sigma(voltage_kv)
    psi0 = shift_beam_fourier(beam, positions, real_space_calib_ang, dtype)
    dpsi0 = shift_beam_fourier(db, positions, real_space_calib_ang, dtype)
    prop = propagation_func(beam.shape[0], beam.shape[1], slice_thickness, voltage_kv, calib, dtype)
    num = slices.shape[2]
    data = np.empty((positions.shape[0],) + beam.shape[:2], np.float64)
    ddata = np.empty_like(data)
    for i in range(positions.shape[0]):
        wave, dwave = psi0[i], dpsi0[i]
        for s in range(num):
            trans = transmission_func(slices[:, :, s], voltage_kv, dtype)[..., None]
            dwave = trans * (dwave + 1j * sigma * dsl[:, :, s][..., None] * wave)
            wave = wave * trans
            if s != num - 1:
                wave = np.fft.ifft2(np.fft.fft2(wave, axes=(0, 1)) * prop[..., None], axes=(0, 1))
                dwave = np.fft.ifft2(np.fft.fft2(dwave, axes=(0, 1)) * prop[..., None], axes=(0, 1))
        amp = np.fft.fftshift(np.fft.fft2(wave, axes=(0, 1)), axes=(0, 1))
        damp = np.fft.fftshift(np.fft.fft2(dwave, axes=(0, 1)), axes=(0, 1))
        data[i] = np.einsum("m,hwm->hw", w, np.abs(amp) ** 2)
        ddata[i] = np.einsum("m,hwm->hw", w, 2.0 * np.real(np.conj(amp) * damp))
    return data, ddata


# ---------------------------------------------------------------------------
# Ensemble axes: cbed_image's ensemble branch (simulations.py:1163-1193) with
# bind_cbed_axes (:769-888), _apply_tilt_phase_ramp (:891-946) and
# apply_distributions (multislice/reduce.py:92-201); the Gauss-Hermite producers
# of multislice/producers.py:46-290. An axis is (samples (N, D), weights (N,),
# reduction "coherent" | "incoherent", axis_id).
# ---------------------------------------------------------------------------


def gauss_hermite_normal(n_quad):
    x, w = np.polynomial.hermite.hermgauss(int(n_quad))
    return np.sqrt(2.0) * x, w / np.sqrt(np.pi)


def jitter_axis(sigma_ang, n_quad):
    nodes, weights = gauss_hermite_normal(n_quad)
    d = sigma_ang * nodes if sigma_ang > 0 else np.zeros_like(nodes)
    dy, dx = np.meshgrid(d, d, indexing="ij")
    wy, wx = np.meshgrid(weights, weights, indexing="ij")
    w = (wy * wx).reshape(-1)
    return np.stack((dy.reshape(-1), dx.reshape(-1)), axis=1), w / w.sum(), "incoherent", "position_jitter"


def coherence_axis(energy_spread_ev, divergence_mrad, n_quad):
    nodes, weights = gauss_hermite_normal(n_quad)
    e = energy_spread_ev * nodes if energy_spread_ev > 0 else np.zeros_like(nodes)
    t = divergence_mrad * nodes if divergence_mrad > 0 else np.zeros_like(nodes)
    eg, txg, tyg = np.meshgrid(e, t, t, indexing="ij")
    we, wx, wy = np.meshgrid(weights, weights, weights, indexing="ij")
    w = (we * wx * wy).reshape(-1)
    samples = np.stack((eg.reshape(-1), txg.reshape(-1), tyg.reshape(-1)), axis=1)
    return samples, w / w.sum(), "incoherent", "coherence"


def tilt_phase_ramp(modes, tilt_mrad, voltage_kv, calib_ang):
    h, w = modes.shape[0], modes.shape[1]
    y = (np.arange(h, dtype=np.float64) - (h - 1) / 2.0) * calib_ang
    x = (np.arange(w, dtype=np.float64) - (w - 1) / 2.0) * calib_ang
    yy, xx = np.meshgrid(y, x, indexing="ij")
    phase = (2.0 * np.pi / relativistic_wavelength_ang(voltage_kv)) * (
        tilt_mrad[0] / 1000.0 * xx + tilt_mrad[1] / 1000.0 * yy)
    return modes * np.exp(1j * phase)[..., None]


def ensemble_cbed(slices, slice_thickness, pot_calib, beam_modes, beam_calib, voltage_kv, axes):
    """CBED intensity of an ensemble: beam_modes (H, W, M) already at its place."""
    beam_modes = np.atleast_3d(np.asarray(beam_modes)).astype(np.complex128)
    calib = min(float(pot_calib), float(beam_calib))
    counts = [a[0].shape[0] for a in axes]
    amps = np.empty(tuple(counts) + beam_modes.shape[:2], np.complex128)
    for idx in np.ndindex(*counts):
        mode, delta, de, tilt = 0, np.zeros(2), 0.0, np.zeros(2)
        for (samples, _, _, axis_id), k in zip(axes, idx):
            row = samples[k]
            if axis_id == "probe_modes":
                mode = int(row[0])
            elif axis_id == "position_jitter":
                delta = delta + row
            else:
                de, tilt = de + row[0], tilt + row[1:3]
        volt = voltage_kv + de / 1000.0
        sel = beam_modes[:, :, mode:mode + 1]
        shifted = shift_beam_fourier(sel, delta[None, :], calib)[0]
        tilted = tilt_phase_ramp(shifted, tilt, volt, calib)
        amps[idx] = cbed_amplitude(slices, slice_thickness, volt, calib, tilted)[..., 0]
    field = amps
    labels = list(range(len(axes)))
    for ax in sorted([i for i, a in enumerate(axes) if a[2] == "coherent"], reverse=True):
        cur = labels.index(ax)
        field = np.sum(np.moveaxis(field, cur, -1) * axes[ax][1], axis=-1)
        labels.pop(cur)
    inten = np.abs(field) ** 2
    for ax in sorted([i for i, a in enumerate(axes) if a[2] == "incoherent"], reverse=True):
        cur = labels.index(ax)
        inten = np.sum(np.moveaxis(inten, cur, -1) * axes[ax][1], axis=-1)
        labels.pop(cur)
    return inten


def stem_4d_ensemble(slices, slice_thickness, pot_calib, beam_modes, beam_calib, voltage_kv, scan_positions_px,
                     real_space_calib_ang, axes):
    """stem_4d whose microscope carries ensemble axes: per position the scan-shifted
    beam through ensemble_cbed (simulations.py:1386-1427)."""
    positions = np.atleast_2d(np.asarray(scan_positions_px, dtype=np.float64))
    shifted = shift_beam_fourier(beam_modes, positions, real_space_calib_ang)
    return np.stack([ensemble_cbed(slices, slice_thickness, pot_calib, shifted[i], beam_calib, voltage_kv, axes)
                     for i in range(positions.shape[0])])


def crystal_potential_slices(positions, atomic_numbers, lattice, atom_potentials, pixel_size, slice_thickness=1.0,
                             repeats=(1, 1, 1), padding=4.0, grid_shape=None):
    """crystal_potential_slices (multislice/atom_potentials.py:1364-1510) given the
    per-element lookup potentials (atomic number -> (H, W), atom at the centre):
    lattice repeats (:1126-1241), z slicing (:684-745), padded grid (:748-823), every
    atom's Fourier sub-pixel shift of its lookup added to its slice (:826-994), crop.
    Returns (h, w, S) float64."""
    positions = np.asarray(positions, np.float64)
    numbers = np.asarray(atomic_numbers)
    reps = list(repeats)
    if any(r > 1 for r in reps):
        ix, iy, iz = np.meshgrid(np.arange(reps[0]), np.arange(reps[1]), np.arange(reps[2]), indexing="ij")
        shifts = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], -1).astype(np.float64) @ np.asarray(lattice)
        positions = (positions[None] + shifts[:, None]).reshape(-1, 3)
        numbers = np.tile(numbers, shifts.shape[0])
    z = positions[:, 2]
    sidx = np.floor((z - z.min()) / slice_thickness).astype(int)
    x, y = positions[:, 0], positions[:, 1]
    x_min, y_min = x.min() - padding, y.min() - padding
    if grid_shape is not None:
        height, width, num_slices = grid_shape
    else:
        width = int(np.ceil((x.max() + padding - x_min) / pixel_size))
        height = int(np.ceil((y.max() + padding - y_min) / pixel_size))
        crop = int(round(padding / pixel_size))
        width, height = max(width, 2 * crop + 1), max(height, 2 * crop + 1)
        num_slices = int(sidx.max()) + 1
    ky = np.fft.fftfreq(height, d=1.0).reshape(-1, 1)
    kx = np.fft.fftfreq(width, d=1.0).reshape(1, -1)
    out = np.zeros((height, width, num_slices))
    spectra = {int(e): np.fft.fft2(np.asarray(p, np.float64)) for e, p in atom_potentials.items()}
    for a in range(positions.shape[0]):
        if not 0 <= sidx[a] < num_slices:
            continue
        sx = (x[a] - x_min) / pixel_size - width / 2.0
        sy = (y[a] - y_min) / pixel_size - height / 2.0
        phase = np.exp(2j * np.pi * (kx * sx + ky * sy))
        out[:, :, sidx[a]] += np.real(np.fft.ifft2(spectra[int(numbers[a])] * phase))
    crop = int(round(padding / pixel_size))
    return out[crop:height - crop, crop:width - crop, :]


def resize_linear_weights(input_size, output_size, antialias=True):
    """jax.image.resize(method="linear") weights along one axis (jax 0.9.2,
    jax/_src/image/scale.py compute_weight_mat): triangle kernel at half-pixel
    centres, widened by the downscale factor, normalised, zero outside the input.
    Returns (input_size, output_size)."""
    inv_scale = input_size / output_size
    kernel_scale = max(inv_scale, 1.0) if antialias else 1.0
    sample_f = (np.arange(output_size) + 0.5) * inv_scale - 0.5
    x = np.abs(sample_f[None, :] - np.arange(input_size, dtype=np.float64)[:, None]) / kernel_scale
    w = np.maximum(0.0, 1.0 - x)
    tot = w.sum(axis=0, keepdims=True)
    w = np.where(np.abs(tot) > 1000.0 * float(np.finfo(np.float32).eps), w / np.where(tot != 0, tot, 1), 0.0)
    return np.where(((sample_f >= -0.5) & (sample_f <= input_size - 0.5))[None, :], w, 0.0)


def clip_cbed(cbed, fourier_calib_inv_ang, voltage_kv, extent_mrad, output_shape):
    """plots/figuring.py:37-117: crop around (h//2, w//2) to ceil(extent / calib) pixels
    each side (clamped), then a linear resize of the axes whose size changes."""
    cbed = np.asarray(cbed, np.float64)
    h, w = cbed.shape
    px = int(np.ceil((extent_mrad / (relativistic_wavelength_ang(voltage_kv) * 1000.0)) / fourier_calib_inv_ang))
    y0, y1 = max(0, h // 2 - px), min(h, h // 2 + px)
    x0, x1 = max(0, w // 2 - px), min(w, w // 2 + px)
    c = cbed[y0:y1, x0:x1]
    if output_shape[0] != c.shape[0]:
        c = resize_linear_weights(c.shape[0], output_shape[0]).T @ c
    if output_shape[1] != c.shape[1]:
        c = c @ resize_linear_weights(c.shape[1], output_shape[1])
    return c


# ---------------------------------------------------------------------------
# Reconstruction loop (multislice/multislice_recon.py:671-1221) with optax 0.2.3's
# Adam restated, for a few iterations in float64: the checker of the engine's loops.
# ---------------------------------------------------------------------------


def _adam_step(g, state, lr, b1=0.9, b2=0.999, eps=1e-8):
    mu = b1 * state["mu"] + (1 - b1) * g
    nu = b2 * state["nu"] + (1 - b2) * np.real(np.conj(g) * g)
    c = state["count"] + 1
    step = -lr * (mu / (1 - b1 ** c)) / (np.sqrt(nu / (1 - b2 ** c)) + eps)
    return step, {"mu": mu, "nu": nu, "count": c}


def single_slice_poscorrected(data, positions, voltage_kv, calib_ang, pot0, beam0, slice_thickness, iterations,
                              lr, lr_pos):
    """MSE loss, one slice; returns (pot, beam, positions, losses)."""
    pot, beam, pos = pot0.astype(np.complex128), beam0.astype(np.complex128), np.asarray(positions, np.float64)
    zero = lambda x: {"mu": np.zeros_like(x), "nu": np.zeros(x.shape), "count": 0}
    s_pot, s_beam, s_pos = zero(pot), zero(beam), zero(pos)
    losses = []
    for _ in range(iterations):
        model = stem_4d(np.real(pot)[..., None], slice_thickness, calib_ang, beam[..., None], [1.0], calib_ang,
                        voltage_kv, pos, calib_ang)["data"]
        diff = model - data
        losses.append(float(np.mean(diff ** 2)))
        g = 2.0 * diff / diff.size
        dv, dbeam, dpos = stem_4d_vjp(np.real(pot)[..., None], slice_thickness, calib_ang, beam[..., None], [1.0],
                                      calib_ang, voltage_kv, pos, calib_ang, g, with_positions=True)
        # the reference steps with conj(JAX gradient)
        step, s_pot = _adam_step(dv[:, :, 0].astype(np.complex128), s_pot, lr)
        pot = pot + step
        step, s_beam = _adam_step(np.conj(dbeam[:, :, 0]), s_beam, lr)
        beam = beam + step
        step, s_pos = _adam_step(dpos, s_pos, lr_pos)
        pos = pos + step
    return pot, beam, pos, losses


def _optax_adam(g, state, lr, b1=0.9, b2=0.999, eps=1e-8):
    """optax 0.2.3 ``adam`` (``scale_by_adam`` then ``scale_by_learning_rate``), in its
    operation order: mu = (1 - b1) g + b1 mu; nu = (1 - b2) |g|^2 + b2 nu; bias
    corrections 1 - b^count; update = -lr * mu_hat / (sqrt(nu_hat) + eps)."""
    sq = np.real(np.conj(g) * g) if np.iscomplexobj(g) else g ** 2
    mu = (1 - b1) * g + b1 * state["mu"]
    nu = (1 - b2) * sq + b2 * state["nu"]
    count = state["count"] + 1
    mu_hat = mu / (1 - b1 ** count)
    nu_hat = nu / (1 - b2 ** count)
    return -lr * (mu_hat / (np.sqrt(nu_hat) + eps)), {"mu": mu, "nu": nu, "count": count}


def _loss_grad(model, data, loss):
    """``_reduce_loss`` (multislice/multislice_recon.py:127-147) and its derivative."""
    diff = model - data
    if loss == "mae":
        return float(np.mean(np.abs(diff))), np.sign(diff) / diff.size
    mse = float(np.mean(diff ** 2))
    if loss == "mse":
        return mse, 2.0 * diff / diff.size
    rmse = np.sqrt(mse)
    return float(rmse), diff / (diff.size * rmse)


def recon_loop(data, positions, voltage_kv, calib_ang, pot0, modes0, weights, slice_thickness, num_iterations,
               lr, lr_pos=None, save_every=1, loss="mse"):
    """The reference's reconstruction loops in float64 with optax's Adam
    (multislice/multislice_recon.py): ``single_slice_ptychography`` (:243-668,
    ``lr_pos`` None: positions fixed), ``single_slice_poscorrected`` (:671-1221),
    ``single_slice_multi_modal`` (:1224-1737; several modes with fixed weights) and
    ``multi_slice_multi_modal`` (:1740-2227) all follow it.

    Each iteration: patterns = stem_4d(real(pot) as one slice, modes, weights,
    positions) (:392-420), the loss of ``_reduce_loss``, JAX's gradients (the VJP of
    ``stem_4d``: dL/dV real, the modes' and positions' gradients), then one optimizer
    step per parameter. Potential and modes step with conj of JAX's gradient
    (``_apply_optimizer_step`` :166-207), positions with their real gradient and
    ``optax.apply_updates``. Snapshots: after the first update at index 0, then after
    iteration ii at index ii // save_every when ii % save_every == 0 (:590-636),
    out-of-range indices dropped. Returns a dict of the final values, snapshots
    (trailing axis) and losses."""
    pot = np.asarray(pot0).astype(np.complex128)
    modes = np.atleast_3d(np.asarray(modes0)).astype(np.complex128)
    w = np.asarray(weights, np.float64)
    pos = np.asarray(positions, np.float64).copy()
    refine = lr_pos is not None
    zero = lambda x: {"mu": np.zeros_like(x), "nu": np.zeros(x.shape), "count": 0}
    s_pot, s_modes, s_pos = zero(pot), zero(modes), zero(pos)
    count = num_iterations // save_every
    snap = {"pot": np.zeros(pot.shape + (count,), np.complex128),
            "modes": np.zeros(modes.shape + (count,), np.complex128),
            "pos": np.zeros(pos.shape + (count,), np.float64)}
    losses = []
    for ii in range(num_iterations):
        slices = np.real(pot)[..., None]
        model = stem_4d(slices, slice_thickness, calib_ang, modes, w, calib_ang, voltage_kv, pos,
                        calib_ang)["data"]
        value, g = _loss_grad(model, np.asarray(data, np.float64), loss)
        losses.append(value)
        out = stem_4d_vjp(slices, slice_thickness, calib_ang, modes, w, calib_ang, voltage_kv, pos, calib_ang, g,
                          with_positions=refine)
        dv, dm = out[0], out[1]
        step, s_pot = _optax_adam(dv[:, :, 0].astype(np.complex128), s_pot, lr)
        pot = pot + step
        step, s_modes = _optax_adam(np.conj(dm), s_modes, lr)
        modes = modes + step
        if refine:
            step, s_pos = _optax_adam(out[2], s_pos, lr_pos)
            pos = pos + step
        if ii % save_every == 0 and ii // save_every < count:
            snap["pot"][..., ii // save_every] = pot
            snap["modes"][..., ii // save_every] = modes
            snap["pos"][..., ii // save_every] = pos
    return {"pot": pot, "modes": modes, "pos": pos, "snap_pot": snap["pot"], "snap_modes": snap["modes"],
            "snap_pos": snap["pos"], "losses": losses}


# ---------------------------------------------------------------------------
# Single-atom projected potentials (multislice/atom_potentials.py:95-681,
# multislice/form_factors.py:322-439), float64.
# ---------------------------------------------------------------------------

def _bessel_k0_ref(x):
    """The reference's K0 (atom_potentials.py:95-140, :377-408): Abramowitz & Stegun
    9.8.5 for x <= 2 (with I0), 9.8.6 above."""
    from scipy.special import i0
    x = np.asarray(x, np.float64)
    x2 = (x * x) / 4.0
    c = np.array([-0.57721566, 0.42278420, 0.23069756, 0.03488590, 0.00262698, 0.00010750, 0.00000740])
    small = -np.log(x / 2.0) * i0(x) + np.sum(c * np.power(x2[..., None], np.arange(7)), axis=-1)
    y = 2.0 / x
    poly = 1.25331414 + y * (-0.07832358 + y * (0.02189568 + y * (-0.01062446 + y * (
        0.00587872 + y * (-0.00251540 + y * 0.00053208)))))
    return np.where(x <= 2.0, small, np.exp(-x) / np.sqrt(x) * poly)


def _bessel_k1_ref(x):
    """The reference's K1 (atom_potentials.py:279-297, :409-421): A&S 9.8.7 for x <= 2
    (with I1), 9.8.8 above."""
    from scipy.special import i1
    x = np.asarray(x, np.float64)
    x2 = (x * x) / 4.0
    d = np.array([1.0, 0.15443144, -0.67278579, -0.18156897, -0.01919402, -0.00110404, -0.00004686])
    small = np.log(x / 2.0) * i1(x) + np.sum(d * np.power(x2[..., None], np.arange(7)), axis=-1) / x
    y = 2.0 / x
    poly = 1.25331414 + y * (0.23498619 + y * (-0.03655620 + y * (0.01504268 + y * (
        -0.00780353 + y * (0.00325614 + y * -0.00068245)))))
    return np.where(x <= 2.0, small, np.exp(-x) / np.sqrt(x) * poly)


def element_coefficients(atom_no, parameterization):
    """Row of the coefficient table the package ships (lobato: a1..a5, b1..b5;
    kirkland: a1, b1, ..., c3, d3)."""
    import os
    data = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ptyrodactyl_b200", "data")
    if parameterization == "lobato":
        tab = np.loadtxt(os.path.join(data, "lobato_van_dyck.csv"), delimiter=",", skiprows=1, usecols=range(2, 12))
    else:
        tab = np.loadtxt(os.path.join(data, "kirkland_potentials.csv"), delimiter=",")
    return tab[int(atom_no) - 1]


def projected_potential(coeffs, r, parameterization):
    """lobato_projected_potential (form_factors.py:322-371, Lobato & Van Dyck Eq. 16,
    C_MB = 47.87801) or kirkland_projected_potential (:374-439, a0 = 0.5292, e_k = 14.4)."""
    r = np.maximum(np.asarray(r, np.float64), 1e-10)[..., None]
    if parameterization == "lobato":
        a, b = np.asarray(coeffs[:5]), np.asarray(coeffs[5:10])
        arg = 2.0 * np.pi * r / np.sqrt(b)
        terms = a / b * _bessel_k0_ref(arg) + a * np.pi * r / np.power(b, 1.5) * _bessel_k1_ref(arg)
        return 2.0 * np.pi * 47.87801 * np.sum(terms, axis=-1)
    c = np.asarray(coeffs)
    la, lb, ga, gb = c[[0, 2, 4]], c[[1, 3, 5]], c[[6, 8, 10]], c[[7, 9, 11]]
    lt = la * _bessel_k0_ref(2.0 * np.pi * r * np.sqrt(lb))
    gt = ga / gb * np.exp(-(np.pi ** 2) * np.square(r) / gb)
    lpre = 4.0 * np.pi ** 2 * 0.5292 * 14.4
    gpre = 2.0 * np.pi ** 2 * 0.5292 * 14.4
    return lpre * (lt[..., 0] + lt[..., 1] + lt[..., 2]) + gpre * (gt[..., 0] + gt[..., 1] + gt[..., 2])


def single_atom_potential(atom_no, pixel_size, grid_shape, center_coords=None, supersampling=4,
                          parameterization="lobato"):
    """atom_potentials.py:588-681: the potential on a supersampled grid (point k of an
    axis at (k - K/2) * pixel / s), r = sqrt(dx^2 + dy^2 + 1e-10), then the mean of each
    pixel's s x s block (``_downsample_potential`` :537-583)."""
    s = int(supersampling)
    step = pixel_size / s
    gh, gw = grid_shape[0] * s, grid_shape[1] * s
    cx, cy = (0.0, 0.0) if center_coords is None else (center_coords[0], center_coords[1])
    yc = (np.arange(gh) - gh // 2) * step
    xc = (np.arange(gw) - gw // 2) * step
    ya, xa = np.meshgrid(yc, xc, indexing="ij")
    r = np.sqrt((xa - cx) ** 2 + (ya - cy) ** 2 + 1e-10)
    fine = projected_potential(element_coefficients(atom_no, parameterization), r, parameterization)
    return fine.reshape(grid_shape[0], s, grid_shape[1], s).mean(axis=(1, 3))
