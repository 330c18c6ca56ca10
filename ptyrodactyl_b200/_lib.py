"""ctypes binding of ``libptyro_b200.so`` (the C-ABI in ``include/ptyro_b200.h``).

The product path has no CPU fallback: if the library is missing or cannot be
loaded this module raises, and every public entry point fails loudly.
"""

from __future__ import annotations

import ctypes
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libptyro_b200.so")

PTYRO_OK = 0
PTYRO_ERR_INVALID = 1
PTYRO_ERR_WORKSPACE = 2
PTYRO_ERR_CUDA = 3
PTYRO_ERR_UNSUPPORTED = 4
STATIC_SCRATCH_BYTES = 64 << 20  # PTYRO_STATIC_SCRATCH_BYTES
WS_STATUS_BYTES = 256  # PTYRO_WS_STATUS_BYTES: the status block at the start of every workspace
STATUS_WAIT_TIMEOUT = 1  # PTYRO_STATUS_WAIT_TIMEOUT
PTYRO_FLAG_ACCUMULATE = 1
MAX_DETECTORS = 32

# every symbol include/ptyro_b200.h declares
EXPORTED_SYMBOLS = (
    "ptyro_version",
    "ptyro_last_error",
    "ptyro_ms_workspace_bytes",
    "ptyro_ms_forward",
    "ptyro_ms_forward_to_host",
    "ptyro_ms_forward_plain",
    "ptyro_make_probe",
    "ptyro_fft_workspace_bytes",
    "ptyro_fft2",
    "ptyro_launch_count",
    "ptyro_pass_wait_timeouts",
    "ptyro_ms_steady_pass",
    "ptyro_fp32_fma_probe",
    "ptyro_test_wait_timeout",
    "ptyro_ms_forward_noalloc",
    "ptyro_ms_detect_workspace_bytes",
    "ptyro_ms_forward_detect",
    "ptyro_detect_patterns",
    "ptyro_detect_patterns_hw",
    "ptyro_ms_jvp_workspace_bytes",
    "ptyro_ms_jvp",
    "ptyro_ms_forward_tilted",
    "ptyro_ms_amplitudes",
    "ptyro_place_atoms_workspace_bytes",
    "ptyro_place_atoms",
    "ptyro_clip_resize_workspace_bytes",
    "ptyro_clip_resize",
    "ptyro_ms_residual_bytes",
    "ptyro_ms_forward_ckpt",
    "ptyro_ms_backward_workspace_bytes",
    "ptyro_ms_backward",
    "ptyro_ms_backward_positions",
    "ptyro_sched_job_bytes",
    "ptyro_sched_create",
    "ptyro_sched_destroy",
    "ptyro_sched_submit",
    "ptyro_sched_cancel",
    "ptyro_sched_step",
    "ptyro_sched_job_state",
    "ptyro_sched_release",
    "ptyro_sched_memory",
    "ptyro_plan_bytes",
    "ptyro_plan_create",
    "ptyro_plan_launch",
    "ptyro_plan_job_status",
    "ptyro_plan_destroy",
    "ptyro_atom_slices_workspace_bytes",
    "ptyro_atom_slices",
    "ptyro_atom_potential",
    "ptyro_ms_weight_grad_workspace_bytes",
    "ptyro_ms_weight_grad",
    "ptyro_gm_workspace_bytes",
    "ptyro_gm_residual_bytes",
    "ptyro_gm_forward",
    "ptyro_gm_backward_workspace_bytes",
    "ptyro_gm_backward",
    "ptyro_gm_jvp_workspace_bytes",
    "ptyro_gm_jvp",
    "ptyro_gm_fft_workspace_bytes",
    "ptyro_gm_fft2",
    "ptyro_gm_make_probe_workspace_bytes",
    "ptyro_gm_make_probe",
    "ptyro_gm_weight_grad_workspace_bytes",
    "ptyro_gm_weight_grad",
)

PTYRO_JOB_FORWARD = 0
PTYRO_JOB_GRADIENT = 1
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4


class MsParams(ctypes.Structure):
    """Mirror of ``ptyro_ms_params``."""

    _fields_ = [
        ("n", ctypes.c_int32),
        ("num_slices", ctypes.c_int32),
        ("num_modes", ctypes.c_int32),
        ("num_probes", ctypes.c_int32),
        ("batch", ctypes.c_int32),
        ("tune", ctypes.c_int32),
        ("field_n", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("voltage_kv", ctypes.c_double),
        ("slice_thickness_ang", ctypes.c_double),
        ("calib_ang", ctypes.c_double),
        ("shift_calib_ang", ctypes.c_double),
        ("pot_stride_y", ctypes.c_int64),
        ("pot_stride_x", ctypes.c_int64),
        ("pot_stride_s", ctypes.c_int64),
        ("mode_stride_y", ctypes.c_int64),
        ("mode_stride_x", ctypes.c_int64),
        ("mode_stride_m", ctypes.c_int64),
        ("windows", ctypes.c_void_p),
    ]


class JobDesc(ctypes.Structure):
    """Mirror of ``ptyro_job_desc``."""

    _fields_ = [
        ("p", MsParams),
        ("kind", ctypes.c_int32),
        ("ckpt_every", ctypes.c_int32),
        ("potential", ctypes.c_void_p),
        ("modes", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
        ("positions", ctypes.c_void_p),
        ("patterns", ctypes.c_void_p),
        ("targets", ctypes.c_void_p),
        ("grad_potential", ctypes.c_void_p),
        ("grad_modes", ctypes.c_void_p),
        ("loss", ctypes.c_void_p),
        ("ready_event", ctypes.c_void_p),
    ]


class PtyroError(RuntimeError):
    """A C-ABI call returned an error code."""

    def __init__(self, code: int, message: str):
        super().__init__(f"ptyro_b200 error {code}: {message}")
        self.code = code


_lock = threading.Lock()
_lib = None


def _declare(lib) -> None:
    vp, sz, i32, dbl = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_double
    pp = ctypes.POINTER(MsParams)
    lib.ptyro_version.restype = ctypes.c_int
    lib.ptyro_version.argtypes = []
    lib.ptyro_last_error.restype = ctypes.c_char_p
    lib.ptyro_last_error.argtypes = []
    lib.ptyro_ms_workspace_bytes.restype = sz
    lib.ptyro_ms_workspace_bytes.argtypes = [pp]
    lib.ptyro_ms_forward_to_host.restype = ctypes.c_int
    lib.ptyro_ms_forward_to_host.argtypes = [pp, vp, vp, vp, vp, vp, vp, vp, sz, vp, vp]
    for name in ("ptyro_ms_forward", "ptyro_ms_forward_plain"):
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = [pp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_make_probe.restype = ctypes.c_int
    lib.ptyro_make_probe.argtypes = [i32, dbl, dbl, dbl, dbl, dbl, dbl, vp, vp, sz, vp]
    lib.ptyro_fft_workspace_bytes.restype = sz
    lib.ptyro_fft_workspace_bytes.argtypes = [i32]
    lib.ptyro_fft2.restype = ctypes.c_int
    lib.ptyro_fft2.argtypes = [i32, i32, i32, vp, vp, sz, vp]
    lib.ptyro_launch_count.restype = ctypes.c_ulonglong
    lib.ptyro_launch_count.argtypes = []
    lib.ptyro_pass_wait_timeouts.restype = ctypes.c_uint
    lib.ptyro_pass_wait_timeouts.argtypes = []
    lib.ptyro_ms_steady_pass.restype = ctypes.c_int
    lib.ptyro_ms_steady_pass.argtypes = [pp, i32, i32, vp, sz, vp]
    lib.ptyro_fp32_fma_probe.restype = ctypes.c_int
    lib.ptyro_fp32_fma_probe.argtypes = [vp, i32, i32, vp]
    lib.ptyro_ms_residual_bytes.restype = sz
    lib.ptyro_ms_residual_bytes.argtypes = [pp, i32]
    lib.ptyro_ms_forward_ckpt.restype = ctypes.c_int
    lib.ptyro_ms_forward_ckpt.argtypes = [pp, i32, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_ms_backward_workspace_bytes.restype = sz
    lib.ptyro_ms_backward_workspace_bytes.argtypes = [pp]
    lib.ptyro_ms_backward.restype = ctypes.c_int
    lib.ptyro_ms_backward.argtypes = [pp, i32, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_ms_backward_positions.restype = ctypes.c_int
    lib.ptyro_ms_backward_positions.argtypes = [pp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    jd = ctypes.POINTER(JobDesc)
    lib.ptyro_sched_job_bytes.restype = sz
    lib.ptyro_sched_job_bytes.argtypes = [jd]
    lib.ptyro_sched_create.restype = ctypes.c_int
    lib.ptyro_sched_create.argtypes = [i32, vp, sz, i32, ctypes.POINTER(vp)]
    lib.ptyro_sched_destroy.restype = ctypes.c_int
    lib.ptyro_sched_destroy.argtypes = [vp]
    lib.ptyro_sched_submit.restype = ctypes.c_int
    lib.ptyro_sched_submit.argtypes = [vp, jd, ctypes.POINTER(ctypes.c_int64)]
    lib.ptyro_sched_cancel.restype = ctypes.c_int
    lib.ptyro_sched_cancel.argtypes = [vp, ctypes.c_int64]
    lib.ptyro_sched_step.restype = ctypes.c_int
    lib.ptyro_sched_step.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32)]
    lib.ptyro_sched_job_state.restype = ctypes.c_int
    lib.ptyro_sched_job_state.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(i32)]
    lib.ptyro_sched_release.restype = ctypes.c_int
    lib.ptyro_sched_release.argtypes = [vp, ctypes.c_int64]
    lib.ptyro_sched_memory.restype = ctypes.c_int
    lib.ptyro_sched_memory.argtypes = [vp, ctypes.POINTER(sz), ctypes.POINTER(i32)]
    lib.ptyro_plan_bytes.restype = sz
    lib.ptyro_plan_bytes.argtypes = [jd, i32]
    lib.ptyro_plan_create.restype = ctypes.c_int
    lib.ptyro_plan_create.argtypes = [i32, jd, i32, vp, sz, ctypes.POINTER(vp)]
    lib.ptyro_plan_launch.restype = ctypes.c_int
    lib.ptyro_plan_launch.argtypes = [vp, vp]
    lib.ptyro_plan_job_status.restype = ctypes.c_int
    lib.ptyro_plan_job_status.argtypes = [vp, i32, ctypes.POINTER(vp)]
    lib.ptyro_plan_destroy.restype = ctypes.c_int
    lib.ptyro_plan_destroy.argtypes = [vp]
    i64 = ctypes.c_int64
    lib.ptyro_ms_detect_workspace_bytes.restype = sz
    lib.ptyro_ms_detect_workspace_bytes.argtypes = [pp, i32]
    lib.ptyro_ms_forward_detect.restype = ctypes.c_int
    lib.ptyro_ms_forward_detect.argtypes = [pp, vp, vp, vp, vp, vp, i32, vp, vp, vp, sz, vp]
    lib.ptyro_detect_patterns.restype = ctypes.c_int
    lib.ptyro_detect_patterns.argtypes = [vp, i64, i32, vp, i32, vp, vp]
    lib.ptyro_detect_patterns_hw.restype = ctypes.c_int
    lib.ptyro_detect_patterns_hw.argtypes = [vp, i64, i32, i32, vp, i32, vp, vp]
    lib.ptyro_ms_jvp_workspace_bytes.restype = sz
    lib.ptyro_ms_jvp_workspace_bytes.argtypes = [pp]
    lib.ptyro_ms_jvp.restype = ctypes.c_int
    lib.ptyro_ms_jvp.argtypes = [pp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_ms_forward_tilted.restype = ctypes.c_int
    lib.ptyro_ms_forward_tilted.argtypes = [pp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_ms_amplitudes.restype = ctypes.c_int
    lib.ptyro_ms_amplitudes.argtypes = [pp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_place_atoms_workspace_bytes.restype = sz
    lib.ptyro_place_atoms_workspace_bytes.argtypes = [i32, i32, i32]
    lib.ptyro_place_atoms.restype = ctypes.c_int
    lib.ptyro_place_atoms.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, i64, i64, i64, vp, sz, vp]
    lib.ptyro_clip_resize_workspace_bytes.restype = sz
    lib.ptyro_clip_resize_workspace_bytes.argtypes = [i64, i32, i32]
    lib.ptyro_clip_resize.restype = ctypes.c_int
    lib.ptyro_clip_resize.argtypes = [vp, i64, i32, i32, i32, i32, i32, i32, vp, i32, vp, i32, vp, vp, sz, vp]
    lib.ptyro_atom_slices_workspace_bytes.restype = sz
    lib.ptyro_atom_slices_workspace_bytes.argtypes = [i32, i32]
    lib.ptyro_atom_slices.restype = ctypes.c_int
    lib.ptyro_atom_slices.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, dbl, vp, i64, i64, i64, vp, sz, vp]
    lib.ptyro_ms_forward_noalloc.restype = ctypes.c_int
    lib.ptyro_ms_forward_noalloc.argtypes = [pp, vp, vp, vp, vp, vp, vp]
    lib.ptyro_test_wait_timeout.restype = ctypes.c_int
    lib.ptyro_test_wait_timeout.argtypes = [i32, i32, vp, vp, vp]
    lib.ptyro_ms_weight_grad_workspace_bytes.restype = sz
    lib.ptyro_ms_weight_grad_workspace_bytes.argtypes = [pp]
    lib.ptyro_ms_weight_grad.restype = ctypes.c_int
    lib.ptyro_ms_weight_grad.argtypes = [pp, i32, vp, vp, vp, vp, sz, vp]
    for name in ("ptyro_gm_workspace_bytes", "ptyro_gm_residual_bytes", "ptyro_gm_backward_workspace_bytes"):
        getattr(lib, name).restype = sz
        getattr(lib, name).argtypes = [pp, i32, i32]
    lib.ptyro_gm_jvp_workspace_bytes.restype = sz
    lib.ptyro_gm_jvp_workspace_bytes.argtypes = [pp, i32, i32]
    lib.ptyro_gm_jvp.restype = ctypes.c_int
    lib.ptyro_gm_jvp.argtypes = [pp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_gm_fft_workspace_bytes.restype = sz
    lib.ptyro_gm_fft_workspace_bytes.argtypes = [i32, i32]
    lib.ptyro_gm_fft2.restype = ctypes.c_int
    lib.ptyro_gm_fft2.argtypes = [i32, i32, i32, i32, vp, vp, sz, vp]
    lib.ptyro_gm_make_probe_workspace_bytes.restype = sz
    lib.ptyro_gm_make_probe_workspace_bytes.argtypes = [i32, i32]
    lib.ptyro_gm_make_probe.restype = ctypes.c_int
    lib.ptyro_gm_make_probe.argtypes = [i32, i32, dbl, dbl, dbl, dbl, dbl, dbl, vp, vp, sz, vp]
    lib.ptyro_gm_weight_grad_workspace_bytes.restype = sz
    lib.ptyro_gm_weight_grad_workspace_bytes.argtypes = [pp, i32, i32]
    lib.ptyro_gm_weight_grad.restype = ctypes.c_int
    lib.ptyro_gm_weight_grad.argtypes = [pp, i32, i32, vp, vp, vp, vp, sz, vp]
    lib.ptyro_gm_forward.restype = ctypes.c_int
    lib.ptyro_gm_forward.argtypes = [pp, i32, i32, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_gm_backward.restype = ctypes.c_int
    lib.ptyro_gm_backward.argtypes = [pp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.ptyro_atom_potential.restype = ctypes.c_int
    lib.ptyro_atom_potential.argtypes = [i32, vp, dbl, i32, i32, dbl, dbl, i32, vp, vp]


def load(path: str | None = None):
    """Load (once) and return the engine library; raise if it is unavailable."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise RuntimeError(
                f"{p} is missing: build the sm_100a engine with "
                "`python -m ptyrodactyl_b200.build` (there is no CPU fallback)")
        lib = ctypes.CDLL(p)
        _declare(lib)
        _lib = lib
        return lib


def check(code: int) -> None:
    """Raise :class:`PtyroError` for a non-zero return code."""
    if code != PTYRO_OK:
        msg = load().ptyro_last_error().decode("utf-8", "replace")
        if code == PTYRO_ERR_INVALID or code == PTYRO_ERR_UNSUPPORTED:
            raise ValueError(msg)
        raise PtyroError(code, msg)


class DeviceStatusError(RuntimeError):
    """A call's kernels reported a failure through its device status word (for
    example a bounded wait for a tile copy gave up); its outputs are invalid."""

    def __init__(self, what: str, status: int):
        reasons = []
        if status & STATUS_WAIT_TIMEOUT:
            reasons.append("a bounded wait for a tile copy (TMA) gave up")
        super().__init__(f"{what}: device status {status:#x} ({'; '.join(reasons) or 'unknown bits'}); "
                         "the results of this call are invalid")
        self.status = status


def new_status(device):
    """A zeroed int32 device word that :func:`gather_status` ORs call statuses into."""
    import torch
    return torch.zeros(1, dtype=torch.int32, device=device)


def gather_status(status, workspace) -> None:
    """OR the status word at the start of ``workspace`` (a uint8 device tensor that a
    call just used) into ``status`` on the current stream, ordered after that call.
    Asynchronous and capturable in a CUDA graph; ``status`` None does nothing."""
    if status is not None:
        status.bitwise_or_(workspace[:4].view(status.dtype))


def check_status(status, what: str) -> None:
    """Wait for the work behind ``status`` and raise :class:`DeviceStatusError` if any
    bit is set (a host synchronisation)."""
    v = int(status.item())
    if v:
        raise DeviceStatusError(what, v)


def check_workspace_status(workspace, what: str) -> None:
    """:func:`check_status` of the status word at the start of ``workspace``."""
    import torch
    v = int(workspace[:4].view(torch.int32).item())
    if v:
        raise DeviceStatusError(what, v)
