"""The no-alloc forward, called through the C-ABI, against the workspace forward.

ptyro_ms_forward_noalloc is for callers that cannot allocate device memory (a host
framework that owns all of it, or code running during CUDA stream capture); its
scratch is a fixed array inside the library. This file runs last so a failure here
does not hide the rest of the suite; it also passes when run on its own.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import multislice_ref as R
from ptyrodactyl_b200 import _lib, synth
from ptyrodactyl_b200.simulations import ms_params

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-5  # relative L2, the tolerance of the float32 parity tests


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    w = synth.CONFIG1
    dev = torch.device("cuda")
    pot = torch.as_tensor(synth.potential_slices(w, num_slices=8), device=dev)
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    weights = torch.ones(1, dtype=torch.float32, device=dev)
    pos = torch.as_tensor(synth.raster_positions(w)[:37], device=dev).contiguous()
    prm = ms_params(w.n, 8, 1, 37, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, pot.stride(),
                    modes.stride(), batch=0)
    return lib, prm, pot, modes, weights, pos


def _workspace_forward(lib, prm, pot, modes, weights, pos):
    out = torch.empty((prm.num_probes, prm.n, prm.n), dtype=torch.float32, device=pot.device)
    nbytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=pot.device)
    rc = lib.ptyro_ms_forward(ctypes.byref(prm), pot.data_ptr(), modes.data_ptr(), weights.data_ptr(),
                              pos.data_ptr(), out.data_ptr(), ws.data_ptr(), nbytes,
                              torch.cuda.current_stream().cuda_stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_workspace_forward_twice(case):
    lib, prm, pot, modes, weights, pos = case
    want = _workspace_forward(lib, prm, pot, modes, weights, pos)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the second call reuses the scratch the first one left behind
        out = torch.full((prm.num_probes, prm.n, prm.n), float("nan"), dtype=torch.float32,
                         device=pot.device)
        rc = lib.ptyro_ms_forward_noalloc(ctypes.byref(prm), pot.data_ptr(), modes.data_ptr(),
                                          weights.data_ptr(), pos.data_ptr(), out.data_ptr(), stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert _rel_l2(got, want) <= TOL_F32


def test_noalloc_rejects_jobs_beyond_its_scratch(case):
    lib, _, _, _, weights, pos = case
    dev = pos.device
    # 1024^2 x 16 slices needs a 128 MiB transmission table: more than the fixed scratch.
    # The buffers are full size so that the call would be well-formed if it ran.
    big_pot = torch.zeros((1024, 1024, 16), dtype=torch.float32, device=dev)
    big_modes = torch.zeros((1024, 1024, 1), dtype=torch.complex64, device=dev)
    big_out = torch.empty((1, 1024, 1024), dtype=torch.float32, device=dev)
    one = pos[:1].contiguous()
    big = ms_params(1024, 16, 1, 1, 200.0, 1.95, 0.1, 0.1, big_pot.stride(), big_modes.stride())
    assert lib.ptyro_ms_workspace_bytes(ctypes.byref(big)) > _lib.STATIC_SCRATCH_BYTES
    rc = lib.ptyro_ms_forward_noalloc(ctypes.byref(big), big_pot.data_ptr(), big_modes.data_ptr(),
                                      weights.data_ptr(), one.data_ptr(), big_out.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PTYRO_ERR_WORKSPACE
    assert "no-alloc forward has a fixed" in lib.ptyro_last_error().decode()


def _case_256(num_slices, num_probes):
    w = synth.CONFIG2
    dev = torch.device("cuda")
    pot = torch.as_tensor(synth.potential_slices(w, num_slices=num_slices), device=dev)
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0, w.defocus_ang, w.c3_ang)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    weights = torch.ones(1, dtype=torch.float32, device=dev)
    pos = torch.as_tensor(synth.raster_positions(w)[::613][:num_probes], device=dev).contiguous()
    from ptyrodactyl_b200.simulations import default_tune
    prm = ms_params(w.n, num_slices, 1, pos.shape[0], w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, pot.stride(),
                    modes.stride(), batch=0, tune=default_tune(w.n))
    return prm, pot, modes, weights, pos


def _noalloc(lib, prm, pot, modes, weights, pos):
    out = torch.full((prm.num_probes, prm.n, prm.n), float("nan"), dtype=torch.float32, device=pot.device)
    rc = lib.ptyro_ms_forward_noalloc(ctypes.byref(prm), pot.data_ptr(), modes.data_ptr(), weights.data_ptr(),
                                      pos.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_default_variant_256_bit_identical(case):
    """The default 256^2 launch variant (TMA column blocks, paired passes, line-pair
    transmission tables) on the static scratch: 8 slices keep every table, and the
    patterns equal the workspace forward's bit for bit, twice, with no wait given up."""
    lib = case[0]
    prm, pot, modes, weights, pos = _case_256(8, 5)
    assert lib.ptyro_ms_workspace_bytes(ctypes.byref(prm)) <= _lib.STATIC_SCRATCH_BYTES
    want = _workspace_forward(lib, prm, pot, modes, weights, pos)
    t0 = lib.ptyro_pass_wait_timeouts()
    for _ in range(2):
        assert np.array_equal(_noalloc(lib, prm, pot, modes, weights, pos), want)
    assert lib.ptyro_pass_wait_timeouts() == t0


def test_noalloc_runs_the_full_256_workload_depth(case):
    """256^2 with all 50 slices under the default variant: the interleaved tables do not
    fit the fixed scratch, so the call drops them (bit-identical results) instead of
    rejecting the job."""
    lib = case[0]
    prm, pot, modes, weights, pos = _case_256(50, 3)
    one = ms_params(prm.n, prm.num_slices, 1, 1, prm.voltage_kv, prm.slice_thickness_ang, prm.calib_ang,
                    prm.shift_calib_ang, pot.stride(), modes.stride(), batch=1, tune=prm.tune)
    assert lib.ptyro_ms_workspace_bytes(ctypes.byref(one)) > _lib.STATIC_SCRATCH_BYTES
    got = _noalloc(lib, prm, pot, modes, weights, pos)
    want = _workspace_forward(lib, prm, pot, modes, weights, pos)
    assert np.array_equal(got, want)
