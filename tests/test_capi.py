"""C-ABI library: loads, exports every declared symbol, validates before touching a GPU."""

import ctypes
import os
import re

import pytest

from ptyrodactyl_b200 import _lib
from ptyrodactyl_b200.build import build
from ptyrodactyl_b200.simulations import ms_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.load()


def _declared_functions():
    names = []
    for fname in os.listdir(os.path.join(ROOT, "include")):
        if not fname.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fname)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(ptyro_\w+)\s*\(", text)
    return sorted(set(names))


def test_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(declared) <= set(_lib.EXPORTED_SYMBOLS) | set(declared)
    for name in _lib.EXPORTED_SYMBOLS:
        assert name in declared, f"{name} bound in _lib but not declared in include/"


def test_version(lib):
    assert lib.ptyro_version() >= 100


def _p(**kw):
    base = dict(n=128, num_slices=20, num_modes=1, num_probes=256, voltage_kv=300.0, slice_thickness=1.95,
                calib_ang=0.244, shift_calib_ang=0.244)
    base.update(kw)
    return ms_params(**base)


def test_workspace_bytes_scale(lib):
    small = lib.ptyro_ms_workspace_bytes(ctypes.byref(_p(batch=1)))
    big = lib.ptyro_ms_workspace_bytes(ctypes.byref(_p(batch=16)))
    assert small > 0 and big > small
    assert (big - small) >= 15 * 128 * 128 * 8
    assert lib.ptyro_ms_workspace_bytes(ctypes.byref(_p(n=100))) == 0


@pytest.mark.parametrize("kw,msg", [
    (dict(n=100), "power of two"),
    (dict(n=2048), "power of two"),
    (dict(num_slices=0), "num_slices"),
    (dict(num_modes=0), "num_modes"),
    (dict(voltage_kv=-1.0), "voltage_kv"),
    (dict(slice_thickness=0.0), "slice_thickness"),
    (dict(calib_ang=float("nan")), "calib"),
])
def test_invalid_params_rejected_before_launch(lib, kw, msg):
    p = _p(**kw)
    rc = lib.ptyro_ms_forward(ctypes.byref(p), None, None, None, None, None, None, 0, None)
    assert rc in (_lib.PTYRO_ERR_INVALID, _lib.PTYRO_ERR_UNSUPPORTED)
    assert msg in lib.ptyro_last_error().decode()


def test_workspace_checks(lib):
    p = _p(batch=1)
    buf = ctypes.create_string_buffer(64)
    # null arrays are reported before the workspace
    rc = lib.ptyro_ms_forward(ctypes.byref(p), None, None, None, None, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID
    fake = ctypes.addressof(buf)
    rc = lib.ptyro_ms_forward(ctypes.byref(p), fake, fake, fake, fake, fake, None, 0, None)
    assert rc == _lib.PTYRO_ERR_WORKSPACE
    assert "workspace" in lib.ptyro_last_error().decode()


def test_zero_probes_is_a_no_op(lib):
    p = _p(num_probes=0)
    assert lib.ptyro_ms_forward(ctypes.byref(p), None, None, None, None, None, None, 0, None) == 0


def test_fft2_rejects_bad_edge(lib):
    assert lib.ptyro_fft2(100, 1, 0, None, None, 0, None) == _lib.PTYRO_ERR_UNSUPPORTED
    assert lib.ptyro_fft2(64, -1, 0, None, None, 0, None) == _lib.PTYRO_ERR_INVALID


def test_atom_slices_validate_before_launch(lib):
    ws = lib.ptyro_atom_slices_workspace_bytes(64, 2)
    assert ws > 0
    args = dict(n=64, na=3, nt=2, ns=2, calib=0.2)

    def call(**kw):
        a = {**args, **kw}
        z = ctypes.c_void_p(16)
        return lib.ptyro_atom_slices(a["n"], a["na"], a["nt"], a["ns"], z, z, z, z, None, a["calib"], z,
                                     64 * 2, 2, 1, z, kw.get("wsb", ws), None)

    assert call(n=100) == _lib.PTYRO_ERR_UNSUPPORTED
    assert call(nt=0) == _lib.PTYRO_ERR_INVALID
    assert call(ns=0) == _lib.PTYRO_ERR_INVALID
    assert call(calib=0.0) == _lib.PTYRO_ERR_INVALID
    assert call(wsb=ws - 1) == _lib.PTYRO_ERR_WORKSPACE


def test_atomic_slice_data_validation():
    import numpy as np
    import ptyrodactyl_b200 as pb
    coords = np.zeros((4, 3))
    pots = np.zeros((2, 16, 16))
    ok = pb.create_atomic_slice_data(coords, [0, 1, 0, 1], [[0, 1], [1, 2]], pots)
    assert ok.atom_types.dtype.is_floating_point is False and ok.atom_mask is None
    bad = [
        (dict(atom_coords=np.zeros((4, 2))), "atom_coords must have shape"),
        (dict(atom_types=[0, 1, 0]), "atom_types must have shape"),
        (dict(slice_z_bounds=[0, 1]), "slice_z_bounds must have shape"),
        (dict(atom_potentials=np.zeros((16, 16))), "atom_potentials must have shape"),
        (dict(atom_types=[0, 1, 0, 2]), "atom_types must index atom_potentials"),
        (dict(atom_types=[0, -1, 0, 1]), "atom_types must be non-negative"),
        (dict(slice_z_bounds=[[0, 1], [2, 2]]), "thicknesses must be positive"),
        (dict(atom_coords=np.full((4, 3), np.nan)), "atom_coords contain non-finite"),
        (dict(atom_mask=[1, 1, 0]), "atom_mask must have shape"),
        (dict(atom_mask=[1, np.inf, 0, 1]), "atom_mask contains non-finite"),
    ]
    base = dict(atom_coords=coords, atom_types=[0, 1, 0, 1], slice_z_bounds=[[0, 1], [1, 2]], atom_potentials=pots)
    for kw, msg in bad:
        with pytest.raises(ValueError, match=msg):
            pb.create_atomic_slice_data(**{**base, **kw})


def test_device_status_host_logic():
    """Status words are ORed per call and any set bit raises (host side, no GPU)."""
    import torch
    st = torch.zeros(1, dtype=torch.int32)
    ws = torch.zeros(_lib.WS_STATUS_BYTES, dtype=torch.uint8)
    _lib.gather_status(st, ws)
    _lib.check_status(st, "clean")
    ws[:4] = torch.tensor([_lib.STATUS_WAIT_TIMEOUT, 0, 0, 0], dtype=torch.uint8)
    _lib.gather_status(st, ws)
    _lib.gather_status(None, ws)  # no status tensor: nothing to do
    with pytest.raises(_lib.DeviceStatusError, match="bounded wait"):
        _lib.check_status(st, "failed")
    with pytest.raises(_lib.DeviceStatusError):
        _lib.check_workspace_status(ws, "failed")


def test_any_size_entry_points_validate_before_launch(lib):
    p = _p(n=0, num_probes=4, num_modes=2, num_slices=3)
    ws = lib.ptyro_gm_workspace_bytes(ctypes.byref(p), 45, 77)
    assert ws > 0
    assert lib.ptyro_gm_backward_workspace_bytes(ctypes.byref(p), 45, 77) > ws  # plus the beam sum
    assert lib.ptyro_gm_residual_bytes(ctypes.byref(p), 45, 77) == 8 * 45 * 77 * 4 * 2 * 4
    for h, w in ((0, 77), (45, 0), (4097, 3), (3, 4097)):
        assert lib.ptyro_gm_workspace_bytes(ctypes.byref(p), h, w) == 0
    rc = lib.ptyro_gm_forward(ctypes.byref(p), 45, 77, None, None, None, None, None, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID and "NULL" in lib.ptyro_last_error().decode()
    buf = ctypes.create_string_buffer(64)
    fake = ctypes.addressof(buf)
    rc = lib.ptyro_gm_forward(ctypes.byref(p), 45, 77, fake, fake, fake, fake, fake, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_WORKSPACE
    p.windows = fake
    rc = lib.ptyro_gm_forward(ctypes.byref(p), 45, 77, fake, fake, fake, fake, fake, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_UNSUPPORTED and "windows" in lib.ptyro_last_error().decode()
    p.windows = None
    assert lib.ptyro_gm_forward(ctypes.byref(_p(n=0, num_probes=0)), 45, 77, None, None, None, None, None, None,
                                None, 0, None) == 0
    rc = lib.ptyro_gm_backward(ctypes.byref(p), 45, 77, None, None, None, None, None, None, None, None, None,
                               None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID
    rc = lib.ptyro_gm_weight_grad(ctypes.byref(p), 45, 77, None, None, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID


def test_any_size_jvp_validates(lib):
    p = _p(n=0, num_probes=3, num_modes=1, num_slices=2)
    assert lib.ptyro_gm_jvp_workspace_bytes(ctypes.byref(p), 45, 77) > lib.ptyro_gm_workspace_bytes(
        ctypes.byref(p), 45, 77)
    assert lib.ptyro_gm_jvp_workspace_bytes(ctypes.byref(p), 0, 77) == 0
    rc = lib.ptyro_gm_jvp(ctypes.byref(p), 45, 77, *([None] * 8), None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID and "NULL" in lib.ptyro_last_error().decode()


def test_any_size_transforms_and_probe_validate(lib):
    assert lib.ptyro_gm_fft_workspace_bytes(45, 77) > 0
    assert lib.ptyro_gm_fft_workspace_bytes(0, 77) == 0
    assert lib.ptyro_gm_fft2(4097, 3, 1, 0, None, None, 0, None) == _lib.PTYRO_ERR_INVALID
    assert lib.ptyro_gm_fft2(5, 3, -1, 0, None, None, 0, None) == _lib.PTYRO_ERR_INVALID
    assert lib.ptyro_gm_fft2(5, 3, 0, 0, None, None, 0, None) == 0  # nothing to transform
    assert lib.ptyro_gm_make_probe_workspace_bytes(7, 5) > 0
    rc = lib.ptyro_gm_make_probe(7, 5, -1.0, 25.0, 30.0, 0.0, 0.0, 0.0, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID and "voltage" in lib.ptyro_last_error().decode()
    rc = lib.ptyro_gm_make_probe(7, 5, 200.0, 25.0, 30.0, float("inf"), 0.0, 0.0, None, None, 0, None)
    assert rc == _lib.PTYRO_ERR_INVALID


def test_any_size_routing_host_logic():
    import torch

    from ptyrodactyl_b200.simulations import check_any_grid, engine_grid
    assert engine_grid(64, 64) and engine_grid(1024, 1024)
    for h, w in ((64, 128), (4, 4), (100, 100), (2048, 2048), (45, 77)):
        assert not engine_grid(h, w)
    sl, md = torch.zeros(45, 77, 2), torch.zeros(45, 77, 1, dtype=torch.complex64)
    assert check_any_grid(sl, md) == (45, 77)
    with pytest.raises(ValueError, match="windows"):
        check_any_grid(sl, md, torch.zeros(1, 2, dtype=torch.int32))
    with pytest.raises(ValueError, match="cover the beam grid"):
        check_any_grid(torch.zeros(45, 78, 2), md)
    with pytest.raises(ValueError, match="4096"):
        check_any_grid(torch.zeros(5000, 3, 1), torch.zeros(5000, 3, 1, dtype=torch.complex64))


def test_batch_plan_bytes_validate(lib):
    p = _p(num_probes=5, num_slices=4, batch=2)
    jobs = (_lib.JobDesc * 2)()
    buf = ctypes.create_string_buffer(64)
    fake = ctypes.addressof(buf)
    for j in jobs:
        j.p = p
        j.kind = _lib.PTYRO_JOB_FORWARD
        j.potential = j.modes = j.weights = j.positions = j.patterns = fake
    assert lib.ptyro_plan_bytes(jobs, 2) >= 2 * lib.ptyro_sched_job_bytes(ctypes.byref(jobs[0]))
    assert lib.ptyro_plan_bytes(jobs, 0) == 0
    jobs[1].ready_event = fake  # plans order their inputs on the launch stream
    assert lib.ptyro_plan_bytes(jobs, 2) == 0 and "ready" in lib.ptyro_last_error().decode()
    jobs[1].ready_event = None
    jobs[1].kind = _lib.PTYRO_JOB_GRADIENT  # without targets and gradient buffers
    assert lib.ptyro_plan_bytes(jobs, 2) == 0


def test_forward_to_host_validates_before_launch(lib):
    p = _p(num_probes=4)
    buf = ctypes.create_string_buffer(64)
    fake = ctypes.addressof(buf)
    args = [fake] * 5
    rc = lib.ptyro_ms_forward_to_host(ctypes.byref(p), *args, None, fake, 64, fake, fake + 8)
    assert rc == _lib.PTYRO_ERR_INVALID and "host_patterns" in lib.ptyro_last_error().decode()
    rc = lib.ptyro_ms_forward_to_host(ctypes.byref(p), *args, fake, fake, 64, fake, fake)
    assert rc == _lib.PTYRO_ERR_INVALID and "copy_stream" in lib.ptyro_last_error().decode()
    rc = lib.ptyro_ms_forward_to_host(ctypes.byref(p), *args, fake, fake, 64, fake, None)
    assert rc == _lib.PTYRO_ERR_INVALID
    acc = _p(num_probes=4, flags=_lib.PTYRO_FLAG_ACCUMULATE)
    rc = lib.ptyro_ms_forward_to_host(ctypes.byref(acc), *args, fake, fake, 64, fake, fake + 8)
    assert rc == _lib.PTYRO_ERR_INVALID and "accumulating" in lib.ptyro_last_error().decode()


def test_detect_patterns_hw_validates_before_launch(lib):
    call = lib.ptyro_detect_patterns_hw
    assert call(None, 4, 0, 8, None, 1, None, None) == _lib.PTYRO_ERR_INVALID
    assert call(None, 4, 8, 8193, None, 1, None, None) == _lib.PTYRO_ERR_INVALID
    assert call(None, 4, 8, 8, None, 0, None, None) == _lib.PTYRO_ERR_INVALID
    assert call(None, 4, 8, 8, None, _lib.MAX_DETECTORS + 1, None, None) == _lib.PTYRO_ERR_INVALID
    assert call(None, -1, 8, 8, None, 1, None, None) == _lib.PTYRO_ERR_INVALID
    assert call(None, 0, 7, 5, None, 1, None, None) == _lib.PTYRO_OK
    rc = call(None, 3, 7, 5, None, 1, None, None)
    assert rc == _lib.PTYRO_ERR_INVALID and "NULL" in lib.ptyro_last_error().decode()


def test_stored_mask_bits_is_the_reference_mask():
    """Shifted-order bits for any (H, W): bit d is the reference's annulus d."""
    import numpy as np
    from ptyrodactyl_b200 import detectors as D
    annuli = [(0.0, 5.0), (5.0, 12.0)]
    for shape in [(7, 5), (48, 80), (16, 16)]:
        bits = D.np.zeros(shape, dtype=np.uint32)
        for d, (a, b) in enumerate(annuli):
            bits |= D.annular_mask(shape, 0.05, 200.0, a, b).astype(np.uint32) << np.uint32(d)
        qy = np.arange(shape[0]) - shape[0] // 2
        qx = np.arange(shape[1]) - shape[1] // 2
        q = np.hypot(qy[:, None], qx[None, :]) * 0.05
        lam = D.relativistic_wavelength_ang(200.0)
        assert np.array_equal(bits & 1, ((q >= 0.0) & (q <= 5e-3 / lam)).astype(np.uint32))
