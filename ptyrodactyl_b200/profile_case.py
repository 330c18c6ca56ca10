"""A small, self-checking case of the forward engine for profilers.

    python -m ptyrodactyl_b200.profile_case [n] [probes] [reps] [tune]

Runs one batched forward over ``probes`` scan positions of the perovskite workload
(n x n grid, 2 slices, one batch), then ``reps`` steady-state passes per axis
(``ptyro_ms_steady_pass``) on the wave slots the forward left in the workspace.
Pass-kernel launches: 6 in the forward (setup kernels aside), then ``reps`` row
passes and ``reps`` column passes. Exits non-zero if the patterns are not finite.
"""

from __future__ import annotations

import ctypes
import sys

import torch

from . import _lib, synth
from .simulations import make_probe, ms_params
from .types import create_detector_config, create_microscope_config


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    n = int(argv[0]) if len(argv) > 0 else 256
    probes = int(argv[1]) if len(argv) > 1 else 256
    reps = int(argv[2]) if len(argv) > 2 else 1
    tune = int(argv[3]) if len(argv) > 3 else 3
    w = synth.CONFIG2
    dev = torch.device("cuda")
    lib = _lib.load()
    if n == w.n:
        pot = torch.as_tensor(synth.potential_slices(w, num_slices=2), device=dev)
    else:
        pot = torch.rand((n, n, 2), generator=torch.Generator(device=dev).manual_seed(1), device=dev) * 50
    mic = create_microscope_config(w.voltage_kv, w.aperture_mrad, probe_shape=(n, n))
    det = create_detector_config(w.calib)
    probe = make_probe(mic, det)[..., None].contiguous()
    pos = torch.as_tensor(synth.raster_positions(w), device=dev)[:probes].contiguous()
    probes = pos.shape[0]
    wt = torch.ones(1, device=dev)
    prm = ms_params(n, 2, 1, probes, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, pot.stride(), probe.stride(),
                    probes, tune)
    nb = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    out = torch.empty((probes, n, n), device=dev)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.ptyro_ms_forward(ctypes.byref(prm), pot.data_ptr(), probe.data_ptr(), wt.data_ptr(),
                                    pos.data_ptr(), out.data_ptr(), ws.data_ptr(), nb, st))
    for axis in (0, 1):
        _lib.check(lib.ptyro_ms_steady_pass(ctypes.byref(prm), axis, reps, ws.data_ptr(), nb, st))
    torch.cuda.synchronize()
    total = float(out.sum())
    print(f"profile case n={n} probes={probes} reps={reps} tune={tune}: pattern sum {total:.6g}")
    return 0 if total == total and abs(total) != float("inf") else 1


if __name__ == "__main__":
    sys.exit(main())
