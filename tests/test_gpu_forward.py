"""GPU parity of the forward model against the oracle and the reference's golden vectors.

Tolerances (relative L2 over all pattern values): <= 1e-5 against the float32
(complex64) restatement of the reference; <= 1e-4 against the float64 oracle
and the reference's own float64 golden arrays. The full-depth 512^2 / 100-slice
case is held to 1.5e-5 against the float32 restatement, whose own distance from
float64 is 1e-5 there, and to a smaller float64 error than that restatement.
"""

import ctypes

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from ptyrodactyl_b200 import synth
from ptyrodactyl_b200.simulations import default_tune
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-5
TOL_F64 = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pb._lib.load()


def _run(pot, dz, probe_modes, weights, pos, kv, calib, shift_calib=None, batch=0, plain=False):
    dev = torch.device("cuda")
    slices = torch.as_tensor(np.asarray(pot, np.float32), device=dev)
    modes = torch.as_tensor(np.asarray(probe_modes, np.complex64), device=dev)
    w = torch.as_tensor(np.asarray(weights, np.float32), device=dev)
    p = torch.as_tensor(np.asarray(pos, np.float64), device=dev).reshape(-1, 2).contiguous()
    out = pb.run_forward(slices, dz, modes, w, p, kv, calib, shift_calib or calib, batch=batch, plain=plain)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512, 1024])
def test_fft2_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = (rng.normal(size=(3, n, n)) + 1j * rng.normal(size=(3, n, n))).astype(np.complex64)
    xf = pb.fft2(torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert rel_l2(xf, np.fft.fft2(x.astype(np.complex128))) < 2e-6
    xi = pb.fft2(torch.as_tensor(x, device="cuda"), inverse=True).cpu().numpy()
    assert rel_l2(xi, np.fft.ifft2(x.astype(np.complex128))) < 2e-6


@pytest.mark.parametrize("w", [synth.CONFIG1, synth.CONFIG2])
def test_make_probe_matches_oracle(w):
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, w.defocus_ang, w.c3_ang,
                                      probe_shape=(w.n, w.n))
    det = pb.create_detector_config(w.calib)
    got = pb.make_probe(mic, det).cpu().numpy()
    want = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0, w.defocus_ang, w.c3_ang)
    assert rel_l2(got, want) < 1e-6


def test_reference_golden_plan01(golden):
    g = golden
    probe = R.make_probe(100.0, 20.0, (32, 32), 20.0)
    got = _run(g["pot"], 2.0, probe[..., None], [1.0], g["positions_px"], 100.0, 0.2)
    assert rel_l2(got, g["stem4d"]) < TOL_F64
    # the public API end to end
    slices = pb.create_potential_slices(g["pot"], 2.0, 0.2)
    mic = pb.create_microscope_config(100.0, 20.0, probe_shape=(32, 32))
    det = pb.create_detector_config(0.2, 20.0, scan_positions_px=g["positions_px"])
    beam = pb.create_probe_modes(pb.make_probe(mic, det).cpu().numpy()[..., None], [1.0], 0.2)
    s4 = pb.stem_4d(slices, beam, mic, det)
    assert rel_l2(s4.data.cpu().numpy(), g["stem4d"]) < TOL_F64
    assert np.allclose(s4.scan_positions.cpu().numpy(), g["positions_px"] * 0.2)
    assert abs(s4.fourier_space_calib - 1.0 / (32 * 0.2)) < 1e-12
    cb = pb.cbed_image(slices, beam, mic)
    assert rel_l2(cb.data_array.cpu().numpy(), g["cbed"]) < TOL_F64


def _workload_case(w, n_probes, num_slices=None, seed=0):
    pot = synth.potential_slices(w, num_slices=num_slices)
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0, w.defocus_ang, w.c3_ang)
    pos = synth.raster_positions(w)
    rng = np.random.default_rng(seed)
    pos = pos[rng.choice(pos.shape[0], n_probes, replace=False)]
    return pot, probe, pos


@pytest.mark.parametrize("w,n_probes,num_slices", [(synth.CONFIG1, 6, None), (synth.CONFIG2, 3, 12),
                                                   (synth.CONFIG3, 1, 6)])
def test_forward_matches_oracle(w, n_probes, num_slices):
    pot, probe, pos = _workload_case(w, n_probes, num_slices)
    s = pot.shape[2]
    got = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib)
    args = (pot, synth.SLICE_DZ, w.calib, probe[..., None], [1.0], w.calib, w.voltage_kv, pos, w.calib)
    want32 = R.stem_4d(*args, dtype=np.complex64)["data"]
    want64 = R.stem_4d(*args, dtype=np.complex128)["data"]
    assert rel_l2(got, want32) < TOL_F32, (s, rel_l2(got, want32))
    assert rel_l2(got, want64) < TOL_F64
    n_ap = R.aperture_count(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0)
    assert np.allclose(got.sum(axis=(1, 2)), n_ap, rtol=1e-4)


def _spread_positions(w, count):
    """``count`` raster positions spread over the whole scan (first, last and evenly between)."""
    pos = synth.raster_positions(w)
    return pos[np.linspace(0, pos.shape[0] - 1, count).round().astype(int)]


# At 512^2 and 100 slices the float32 restatement of the reference is itself
# 0.99e-5 - 1.01e-5 (relative L2) away from the float64 oracle, most of it a coherent
# loss of intensity (-8.4e-6) in its own float32 FFTs, so no implementation can be
# within 1e-5 of it without sharing its rounding. There the kernels are held to being
# closer to float64 than that float32 path is, and within 1.5e-5 of it.
TOL_F32_512_100 = 1.5e-5


def _check_full_depth(w, got, pot, probe, pos, tol32=TOL_F32):
    args = (pot, synth.SLICE_DZ, w.calib, probe[..., None], [1.0], w.calib, w.voltage_kv, pos, w.calib)
    want32 = R.stem_4d(*args, dtype=np.complex64)["data"]
    want64 = R.stem_4d(*args, dtype=np.complex128)["data"]
    e32, e64, ref32 = rel_l2(got, want32), rel_l2(got, want64), rel_l2(want32, want64)
    # the kernels against the float32 restatement of the reference, and both against float64
    assert e32 < tol32, (pot.shape[2], e32, e64, ref32)
    assert e64 < TOL_F64, (e64, ref32)
    # the kernels are at least as accurate as the reference's own float32 path
    assert e64 < ref32, (e64, ref32)
    # no coherent loss of intensity: every exact pattern sums to the aperture pixel count
    n_ap = R.aperture_count(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0)
    assert np.allclose(got.sum(axis=(1, 2)), n_ap, rtol=5e-6), got.sum(axis=(1, 2)) / n_ap - 1
    return want64


def test_forward_full_depth_256_50_slices():
    """The 256^2 workload at all 50 slices: 6 probes from corner to corner of the 64 x 64 scan."""
    w = synth.CONFIG2
    pot = synth.potential_slices(w)
    assert pot.shape[2] == 50
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0, w.defocus_ang, w.c3_ang)
    pos = _spread_positions(w, 6)
    got = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib)
    _check_full_depth(w, got, pot, probe, pos)


def test_forward_full_depth_512_100_slices_frozen_phonons():
    """The 512^2 workload at all 100 slices: each of the 4 frozen-phonon configurations
    for 2 probes, and the 4-configuration mean through the public API."""
    w = synth.CONFIG3
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0, w.defocus_ang, w.c3_ang)
    pos = _spread_positions(w, 2)
    pots, wants = [], []
    for k in range(w.phonon_configs):
        pot = synth.potential_slices(w, phonon=k)
        assert pot.shape[2] == 100
        got = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib)
        wants.append(_check_full_depth(w, got, pot, probe, pos, tol32=TOL_F32_512_100))
        pots.append(pot)
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, probe_shape=(w.n, w.n))
    det = pb.create_detector_config(w.calib, scan_positions_px=pos)
    beam = pb.create_probe_modes(probe[..., None], [1.0], w.calib)
    mean = pb.stem_4d_frozen_phonon([pb.create_potential_slices(p, synth.SLICE_DZ, w.calib) for p in pots], beam,
                                    mic, det).data.cpu().numpy()
    assert rel_l2(mean, np.mean(wants, axis=0)) < TOL_F64


def test_modes_weights_and_single_slice():
    rng = np.random.default_rng(3)
    n = 64
    pot = rng.uniform(0, 40, (n, n, 1))
    p1 = R.make_probe(120.0, 22.0, (n, n), 30.0, defocus_ang=30.0)
    modes = np.stack([p1, np.roll(p1, 3, axis=0) * (0.6 + 0.2j)], axis=-1)
    w = np.array([0.7, 0.3])
    pos = np.array([[0.0, 0.0], [1.3, -2.1], [-4.0, 5.5]])
    got = _run(pot, 2.0, modes, w, pos, 120.0, 0.3)
    want = R.stem_4d(pot, 2.0, 0.3, modes, w, 0.3, 120.0, pos, 0.3, dtype=np.complex128)["data"]
    assert rel_l2(got, want) < TOL_F64


def test_batching_is_exact_and_ragged():
    w = synth.CONFIG1
    pot, probe, pos = _workload_case(w, 7, 5)
    a = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib, batch=0)
    b = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib, batch=3)
    c = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos[2:3], w.voltage_kv, w.calib, batch=1)
    assert np.array_equal(a, b)
    assert np.array_equal(a[2], c[0])


def test_plain_path_matches_fused():
    w = synth.CONFIG1
    pot, probe, pos = _workload_case(w, 3, 6)
    fused = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib)
    plain = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib, plain=True)
    assert rel_l2(plain, fused) < TOL_F32


def test_strided_potential_layouts_agree():
    w = synth.CONFIG1
    pot, probe, pos = _workload_case(w, 2, 4)
    dev = torch.device("cuda")
    a = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], pos, w.voltage_kv, w.calib)
    # (S, H, W) storage viewed as (H, W, S)
    shw = torch.as_tensor(np.ascontiguousarray(np.moveaxis(pot, 2, 0)), device=dev, dtype=torch.float32)
    view = shw.permute(1, 2, 0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    wts = torch.ones(1, device=dev)
    p = torch.as_tensor(pos, device=dev)
    b = pb.run_forward(view, synth.SLICE_DZ, modes, wts, p, w.voltage_kv, w.calib, w.calib).cpu().numpy()
    assert np.array_equal(a, b)


def test_zero_positions_returns_empty():
    w = synth.CONFIG1
    pot, probe, _ = _workload_case(w, 1, 2)
    out = _run(pot, synth.SLICE_DZ, probe[..., None], [1.0], np.zeros((0, 2)), w.voltage_kv, w.calib)
    assert out.shape == (0, w.n, w.n)


def test_errors_raise_value_error():
    slices = pb.create_potential_slices(np.zeros((48, 48, 2)), 1.0, 0.2)
    mic = pb.create_microscope_config(100.0, 20.0, probe_shape=(48, 48))
    det = pb.create_detector_config(0.2, scan_positions_px=np.zeros((1, 2)))
    beam = pb.create_probe_modes(np.ones((48, 48, 1), np.complex64), [1.0], 0.2)
    assert tuple(pb.stem_4d(slices, beam, mic, det).data.shape) == (1, 48, 48)  # any grid runs
    beam64 = pb.create_probe_modes(np.ones((64, 64, 1), np.complex64), [1.0], 0.2)
    with pytest.raises(ValueError):  # a potential smaller than the beam's grid
        pb.stem_4d(slices, beam64, mic, det)
    wide = pb.create_potential_slices(np.zeros((5000, 3, 1)), 1.0, 0.2)
    with pytest.raises(ValueError, match="4096"):
        pb.stem_4d(wide, pb.create_probe_modes(np.ones((5000, 3, 1), np.complex64), [1.0], 0.2), mic, det)
    det2 = pb.create_detector_config(0.2)
    with pytest.raises(ValueError, match="scan_positions_px is required"):
        pb.stem_4d(slices, beam, mic, det2)


def test_frozen_phonon_average_matches_oracle_mean():
    w = synth.CONFIG1
    pots = [synth.potential_slices(w, phonon=k, num_slices=4) for k in range(3)]
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0)
    pos = synth.raster_positions(w)[:5]
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, probe_shape=(w.n, w.n))
    det = pb.create_detector_config(w.calib, scan_positions_px=pos)
    beam = pb.create_probe_modes(probe[..., None], [1.0], w.calib)
    got = pb.stem_4d_frozen_phonon([pb.create_potential_slices(p, synth.SLICE_DZ, w.calib) for p in pots], beam,
                                   mic, det).data.cpu().numpy()
    want = np.mean([R.stem_4d(p, synth.SLICE_DZ, w.calib, probe[..., None], [1.0], w.calib, w.voltage_kv, pos,
                              w.calib)["data"] for p in pots], axis=0)
    assert rel_l2(got, want) < TOL_F64


def test_atom_backed_stem4d_sharded_matches_reference_golden(golden):
    g = golden
    atoms = np.array([[2.0, 2.5, 0.25], [4.5, 5.0, 2.25], [3.0, 4.0, 1.25]])
    sample = pb.create_atomic_slice_data(atoms, [0, 0, 0], [[0.0, 2.0], [2.0, 4.0]], g["pot"][..., 0][None])
    mic = pb.create_microscope_config(100.0, 20.0, probe_shape=(32, 32))
    det = pb.create_detector_config(0.2, 20.0, scan_positions_ang=g["positions_px"] * 0.2)
    beam = pb.create_probe_modes(R.make_probe(100.0, 20.0, (32, 32), 20.0)[..., None], [1.0], 0.2)
    s4 = pb.stem4d_sharded(beam, sample, mic, det)
    assert rel_l2(s4.data.cpu().numpy(), g["stem4d_sharded"]) < TOL_F64
    assert np.allclose(s4.scan_positions.cpu().numpy(), g["positions_px"] * 0.2)


def test_slices_from_atoms_match_oracle():
    rng = np.random.default_rng(12)
    n, calib = 128, 0.25
    atoms = np.column_stack([rng.uniform(-5, 40, 300), rng.uniform(-5, 40, 300), rng.uniform(0, 6, 300)])
    types = rng.integers(0, 3, 300)
    kern = rng.uniform(0, 1, (3, n, n)) * np.exp(-np.hypot(*np.meshgrid(np.fft.fftfreq(n) * n, np.fft.fftfreq(n) * n,
                                                                         indexing="ij")) / 3.0)
    bounds = [[0.0, 2.0], [2.0, 4.0], [4.0, 6.0]]
    mask = (rng.uniform(size=300) > 0.2).astype(np.float32)
    sample = pb.create_atomic_slice_data(atoms, types, bounds, kern, mask)
    got = pb.slices_from_atoms(sample, (n, n), calib).cpu().numpy()
    want = np.stack([R.slice_potential_from_atoms(atoms, types, b[0], b[1], kern, (n, n), calib, mask)
                     for b in bounds], axis=-1)
    assert rel_l2(got, want) < 1e-5


def test_cbed_from_atoms_matches_oracle():
    """cbed_amplitude_from_atoms / cbed_image_from_atoms (parallelized.py:174-347):
    slices from atoms on the device, the unshifted modes through them, the image
    reduced over a mode distribution."""
    rng = np.random.default_rng(13)
    n, calib, kv = 64, 0.25, 200.0
    atoms = np.column_stack([rng.uniform(0, 16, 60), rng.uniform(0, 16, 60), rng.uniform(0, 4, 60)])
    types = rng.integers(0, 2, 60)
    r = np.hypot(*np.meshgrid(np.fft.fftfreq(n) * n, np.fft.fftfreq(n) * n, indexing="ij"))
    kern = np.stack([20.0 * np.exp(-r / 2.0), 35.0 * np.exp(-r / 1.5)])
    bounds = [[0.0, 2.0], [2.0, 4.0]]
    probe = R.make_probe(kv, 25.0, (n, n), calib * 100.0, defocus_ang=-20.0)
    modes = np.stack([probe, np.roll(probe, 3, axis=0) * (0.6 + 0.3j)], -1)
    amps = pb.cbed_amplitude_from_atoms(modes, atoms, types, bounds, kern, kv, calib)
    slices = np.stack([R.slice_potential_from_atoms(atoms, types, b[0], b[1], kern, (n, n), calib)
                       for b in bounds], axis=-1)
    want = R.cbed_amplitude(slices, 2.0, kv, calib, modes)
    assert tuple(amps.shape) == (n, n, 2) and rel_l2(amps.cpu().numpy(), want) < TOL_F64
    dist = pb.create_distribution(np.arange(2.0)[:, None], [0.7, 0.3], pb.ReductionMode.INCOHERENT, "probe_modes")
    img = pb.cbed_image_from_atoms(modes, dist, atoms, types, bounds, kern, kv, calib)
    want_img = 0.7 * np.abs(want[..., 0]) ** 2 + 0.3 * np.abs(want[..., 1]) ** 2
    assert rel_l2(img.cpu().numpy(), want_img) < TOL_F64


def test_stem_4d_streams_patterns_to_host():
    """out= a pinned host tensor: chunked compute with overlapped copies gives the
    device result exactly."""
    rng = np.random.default_rng(4)
    n, s, p = 64, 4, 37
    pot = rng.uniform(0, 30, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 20.0)
    pots = pb.create_potential_slices(torch.as_tensor(pot, dtype=torch.float32), 1.5, 0.2)
    beam = pb.create_probe_modes(probe[..., None], [1.0], 0.2)
    mic = pb.create_microscope_config(200.0, 25.0, probe_shape=(n, n))
    det = pb.create_detector_config(0.2, scan_positions_px=rng.uniform(-2, 2, (p, 2)))
    ref = pb.stem_4d(pots, beam, mic, det).data.cpu()
    host = torch.empty((p, n, n), dtype=torch.float32).pin_memory()
    s4 = pb.stem_4d(pots, beam, mic, det, out=host)
    torch.cuda.synchronize()
    assert s4.data is host and torch.equal(host, ref)
    dev_out = torch.empty((p, n, n), dtype=torch.float32, device="cuda")
    assert torch.equal(pb.stem_4d(pots, beam, mic, det, out=dev_out).data.cpu(), ref)


@pytest.mark.parametrize("n,num_slices", [(16, 1), (32, 3), (64, 2), (64, 7), (128, 1), (128, 20)])
def test_resident_kernel_is_bit_identical_to_the_pass_engine(n, num_slices):
    """The wave-resident kernel (tune bit 32768: one CTA per probe, the wave in shared
    memory across all slices) runs the pass engine's operations in the same order, so
    the patterns match the default variant bit for bit; the oracle checks both."""
    rng = np.random.default_rng(n + num_slices)
    pot = rng.uniform(0, 60, (n, n, num_slices))
    probe = R.make_probe(300.0, 20.0, (n, n), 24.4, defocus_ang=20.0)
    pos = rng.uniform(-3, 3, (37, 2))
    dev = torch.device("cuda")
    args = (torch.as_tensor(pot, dtype=torch.float32, device=dev), synth.SLICE_DZ,
            torch.as_tensor(probe[..., None].astype(np.complex64), device=dev), torch.ones(1, device=dev),
            torch.as_tensor(pos, device=dev), 300.0, 0.244, 0.244)
    engine = pb.run_forward(*args, tune=default_tune(n) & ~32768).cpu().numpy()
    resident = pb.run_forward(*args, tune=default_tune(n) | 32768).cpu().numpy()
    assert np.array_equal(resident, engine)
    # several batches, and accumulation into the output (frozen-phonon averaging)
    small = pb.run_forward(*args, tune=default_tune(n) | 32768, batch=5).cpu().numpy()
    assert np.array_equal(small, engine)
    acc = torch.as_tensor(engine, device=dev).clone()
    pb.run_forward(*args, tune=32768, out=acc, accumulate=True)
    assert np.array_equal(acc.cpu().numpy(), engine + engine)
    want = R.stem_4d(pot, synth.SLICE_DZ, 0.244, probe[..., None], [1.0], 0.244, 300.0, pos, 0.244,
                     dtype=np.complex128)["data"]
    assert rel_l2(resident, want) < TOL_F64


def test_resident_kernel_at_the_128_workload_full_depth():
    """The 128^2 perovskite workload (20 slices, 300 kV, 20 mrad) through the resident
    kernel: bit-identical to the pass engine and within the float32 tolerance of the
    float32 restatement."""
    w = synth.CONFIG1
    pot, probe, pos = _workload_case(w, 6)
    dev = torch.device("cuda")
    args = (torch.as_tensor(pot, dtype=torch.float32, device=dev), synth.SLICE_DZ,
            torch.as_tensor(probe[..., None].astype(np.complex64), device=dev), torch.ones(1, device=dev),
            torch.as_tensor(pos, device=dev), w.voltage_kv, w.calib, w.calib)
    engine = pb.run_forward(*args, tune=default_tune(w.n) & ~32768).cpu().numpy()
    resident = pb.run_forward(*args, tune=default_tune(w.n) | 32768).cpu().numpy()
    assert default_tune(w.n) & 32768  # the 128^2 default runs the resident kernel
    assert np.array_equal(resident, engine)
    want32 = R.stem_4d(pot, synth.SLICE_DZ, w.calib, probe[..., None], [1.0], w.calib, w.voltage_kv, pos, w.calib,
                       dtype=np.complex64)["data"]
    assert rel_l2(resident, want32) < TOL_F32


@pytest.mark.parametrize("n", [64, 128])
def test_forward_to_host_streams_every_batch(n):
    """ptyro_ms_forward_to_host with 5-probe batches (a ragged last batch; the pass
    engine at 64^2, the wave-resident kernel at 128^2) copies every batch's patterns
    to pinned host memory on its copy stream: the host patterns equal the device
    forward's bit for bit once the call's stream is synchronised."""
    import ctypes
    from ptyrodactyl_b200.simulations import default_tune, ms_params, run_forward
    rng = np.random.default_rng(n)
    s, p = 4, 23
    dev = torch.device("cuda")
    slices = torch.as_tensor(rng.uniform(0, 30, (n, n, s)), dtype=torch.float32, device=dev)
    probe = R.make_probe(200.0, 25.0, (n, n), 20.0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    wt = torch.ones(1, device=dev)
    pos = torch.as_tensor(rng.uniform(-2, 2, (p, 2)), dtype=torch.float64, device=dev)
    ref = run_forward(slices, 1.5, modes, wt, pos, 200.0, 0.2, 0.2, lanes=1).cpu()
    lib = pb._lib.load()
    prm = ms_params(n, s, 1, p, 200.0, 1.5, 0.2, 0.2, slices.stride(), modes.stride(), 5, default_tune(n))
    ws_bytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    out = torch.empty((p, n, n), dtype=torch.float32, device=dev)
    host = torch.full((p, n, n), -1.0, dtype=torch.float32).pin_memory()
    st, cp = torch.cuda.Stream(), torch.cuda.Stream()
    pb._lib.check(lib.ptyro_ms_forward_to_host(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(),
                                               wt.data_ptr(), pos.data_ptr(), out.data_ptr(), host.data_ptr(),
                                               ws.data_ptr(), ws_bytes, st.cuda_stream, cp.cuda_stream))
    st.synchronize()  # the call's stream waits for the last copy
    assert torch.equal(host, ref)
    assert int(ws[:4].view(torch.int32).item()) == 0
