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
