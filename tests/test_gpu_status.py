"""The device status word: a bounded tile wait that gives up is reported, not hidden.

The self-test kernel arms an mbarrier for a copy that is never issued, so the wait
runs out after a few polls and takes the pass kernels' give-up path (nothing is in
flight, the GPU context stays usable). Real forwards leave the status word zero.
"""

import ctypes

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from ptyrodactyl_b200 import _lib, synth
from ptyrodactyl_b200.simulations import default_tune, ms_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _lib.load()


@pytest.mark.parametrize("warps,polls", [(1, 1), (4, 8), (8, 64)])
def test_wait_that_runs_out_sets_the_status_and_skips_the_warp(warps, polls):
    lib = _lib.load()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = lib.ptyro_pass_wait_timeouts()
    rc = lib.ptyro_test_wait_timeout(warps, polls, status.data_ptr(), skipped.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.STATUS_WAIT_TIMEOUT
    assert int(skipped.item()) == warps
    with pytest.raises(_lib.DeviceStatusError, match="bounded wait"):
        _lib.check_status(status, "self-test")
    # the give-ups are counted by the self-test's own translation unit, not the passes'
    assert lib.ptyro_pass_wait_timeouts() == t0


def test_self_test_rejects_bad_arguments():
    lib = _lib.load()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for warps, polls in [(0, 1), (33, 1), (1, 0), (1, (1 << 20) + 1)]:
        assert lib.ptyro_test_wait_timeout(warps, polls, status.data_ptr(), skipped.data_ptr(), st) == \
            _lib.PTYRO_ERR_INVALID
    assert lib.ptyro_test_wait_timeout(1, 1, None, skipped.data_ptr(), st) == _lib.PTYRO_ERR_INVALID


def test_forwards_after_a_give_up_report_a_clean_status():
    """After the self-test, the default 256^2 and 512^2 variants (TMA column passes)
    run, match the oracle, and their status words stay zero."""
    lib = _lib.load()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.ptyro_test_wait_timeout(2, 4, status.data_ptr(), skipped.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream))
    for w in (synth.CONFIG2, synth.CONFIG3):
        pot = synth.potential_slices(w, num_slices=3)
        probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0, w.defocus_ang, w.c3_ang)
        pos = synth.raster_positions(w)[:2]
        st = _lib.new_status("cuda")
        got = pb.run_forward(torch.as_tensor(pot, device="cuda"), synth.SLICE_DZ,
                             torch.as_tensor(probe[..., None].astype(np.complex64), device="cuda"),
                             torch.ones(1, device="cuda"), torch.as_tensor(pos, device="cuda"), w.voltage_kv, w.calib,
                             w.calib, status=st)
        _lib.check_status(st, "forward")
        want = R.stem_4d(pot, synth.SLICE_DZ, w.calib, probe[..., None], [1.0], w.calib, w.voltage_kv, pos, w.calib,
                         dtype=np.complex128)["data"]
        got = got.cpu().numpy()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-4


def test_workspace_starts_with_a_zeroed_status_block():
    """Every forward zeroes the status word at the start of its workspace itself."""
    lib = _lib.load()
    w = synth.CONFIG2
    pot = torch.as_tensor(synth.potential_slices(w, num_slices=2), device="cuda")
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device="cuda")
    pos = torch.as_tensor(synth.raster_positions(w)[:1], device="cuda").contiguous()
    prm = ms_params(w.n, 2, 1, 1, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, pot.stride(), modes.stride(),
                    tune=default_tune(w.n))
    nbytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = torch.full((nbytes,), 0xFF, dtype=torch.uint8, device="cuda")  # a dirty status word
    out = torch.empty((1, w.n, w.n), dtype=torch.float32, device="cuda")
    _lib.check(lib.ptyro_ms_forward(ctypes.byref(prm), pot.data_ptr(), modes.data_ptr(),
                                    torch.ones(1, device="cuda").data_ptr(), pos.data_ptr(), out.data_ptr(),
                                    ws.data_ptr(), nbytes, torch.cuda.current_stream().cuda_stream))
    _lib.check_workspace_status(ws, "forward")
