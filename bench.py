#!/usr/bin/env python
"""Benchmark of the batched fused multislice forward model (probe-slice updates/s).

Workload: the 256x256 perovskite configuration — 16x16 ABO3 supercell, 50 slices of
1.95 A, 64x64 raster scan (4096 probes), 200 kV, 25 mrad, C1 = -50 A, Cs = 1 um —
with seeded synthetic inputs (``ptyrodactyl_b200.synth``). One step = one full
``stem_4d`` forward over the 4096 probes (4096 * 50 probe-slice updates).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 launch under torchrun: every rank runs its own 4096-probe shard of a
larger scan (weak scaling, no collective on the data path); timings are taken
on the device with CUDA events and reduced as the max over ranks.
Rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from ptyrodactyl_b200 import synth  # noqa: E402
from ptyrodactyl_b200.simulations import default_tune  # noqa: E402

METRIC = "probe-slice updates/s at 256^2 (batched fused multislice forward, 4096 probes x 50 slices)"
UNIT = "probe-slice updates/s"
WORKLOAD = synth.CONFIG2
L2_FLUSH_BYTES = 256 << 20


# ----------------------------------------------------------------------------- CPU leg
_CPU_STATE = {}


def _cpu_worker(task):
    """Oracle (NumPy complex128 restatement of the reference's x64 path) for some probes."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import multislice_ref as R
    name, idx = task
    w = WORKLOAD
    if "pot" not in _CPU_STATE:
        _CPU_STATE["pot"] = synth.potential_slices(w).astype(np.float64)
        _CPU_STATE["probe"] = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0,
                                           w.defocus_ang, w.c3_ang)
        _CPU_STATE["pos"] = synth.raster_positions(w)
    pos = _CPU_STATE["pos"][np.asarray(idx)]
    args = (_CPU_STATE["pot"], synth.SLICE_DZ, w.calib, _CPU_STATE["probe"][..., None], [1.0], w.calib,
            w.voltage_kv, pos, w.calib)
    if name == "check":  # the checker: the float32 and float64 restatements' patterns
        return (R.stem_4d(*args, dtype=np.complex64)["data"], R.stem_4d(*args, dtype=np.complex128)["data"])
    t0 = time.perf_counter()
    R.stem_4d(*args, dtype=np.complex128)
    return time.perf_counter() - t0


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class CpuOracle:
    """A spawn pool (safe next to CUDA) running the oracle on bounded probe samples."""

    def __init__(self, procs: int):
        self.procs = procs
        self.pool = mp.get_context("spawn").Pool(procs)
        # warm every worker (imports, potential generation) outside any timing
        self.pool.map(_cpu_worker, [("warm", [i]) for i in range(procs)])
        self.next = 0

    def step(self, probes_per_proc: int) -> tuple:
        """Run procs * probes_per_proc probes; return (updates, wall seconds)."""
        tasks = []
        for _ in range(self.procs):
            idx = [(self.next + k) % WORKLOAD.num_probes for k in range(probes_per_proc)]
            self.next += probes_per_proc
            tasks.append(("run", idx))
        t0 = time.perf_counter()
        self.pool.map(_cpu_worker, tasks)
        wall = time.perf_counter() - t0
        return self.procs * probes_per_proc * WORKLOAD.num_slices, wall

    def check(self, idx) -> tuple:
        """Oracle patterns (float32 path, float64 path) of the probes ``idx`` of the workload."""
        return self.pool.apply(_cpu_worker, (("check", list(idx)),))

    def close(self):
        self.pool.close()
        self.pool.join()


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ----------------------------------------------------------------------------- GPU leg
def _events(torch, n):
    return [torch.cuda.Event(enable_timing=True) for _ in range(n)]


def fp32_peak_tflops(torch, lib, dev) -> float:
    """Measured FP32 FMA ceiling of this device (TFLOP/s), best of 3."""
    blocks = torch.cuda.get_device_properties(dev).multi_processor_count * 8
    iters = 4096
    out = torch.empty(blocks * 256, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    lib.ptyro_fp32_fma_probe(out.data_ptr(), blocks, 64, st)
    best = 0.0
    for _ in range(3):
        s, e = _events(torch, 2)
        s.record()
        rc = lib.ptyro_fp32_fma_probe(out.data_ptr(), blocks, iters, st)
        e.record()
        torch.cuda.synchronize()
        assert rc == 0
        flops = blocks * 256.0 * iters * 128 * 2
        best = max(best, flops / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import ptyrodactyl_b200 as pb
    from ptyrodactyl_b200 import _lib
    from ptyrodactyl_b200.simulations import ms_params

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    w = WORKLOAD
    n, S, P = w.n, w.num_slices, w.num_probes
    tune = default_tune(n) if args.tune < 0 else args.tune

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuOracle(min(_host_cores(), 64))

    # ---- inputs (this rank's shard: the raster offset by a sub-pixel amount per rank)
    pot = synth.potential_slices(w)
    pos = synth.raster_positions(w) + 0.37 * rank
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, w.defocus_ang, w.c3_ang,
                                      probe_shape=(n, n))
    det = pb.create_detector_config(w.calib, scan_positions_px=pos)
    probe = pb.make_probe(mic, det)
    slices_d = torch.as_tensor(pot, device=dev)
    modes_d = probe[..., None].contiguous()
    weights_d = torch.ones(1, dtype=torch.float32, device=dev)
    pos_d = torch.as_tensor(pos, dtype=torch.float64, device=dev)
    out_d = torch.empty((P, n, n), dtype=torch.float32, device=dev)
    prm = ms_params(n, S, 1, P, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, slices_d.stride(),
                    modes_d.stride(), args.batch, tune)
    ws_bytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        rc = lib.ptyro_ms_forward(ctypes.byref(prm), slices_d.data_ptr(), modes_d.data_ptr(),
                                  weights_d.data_ptr(), pos_d.data_ptr(), out_d.data_ptr(), ws.data_ptr(),
                                  ws_bytes, stream.cuda_stream)
        _lib.check(rc)

    graphed = None
    if args.graph:
        # the same forward captured once as a CUDA graph; a step is one replay
        from ptyrodactyl_b200.graphs import GraphedForward
        graphed = GraphedForward(slices_d, modes_d, weights_d, pos_d, synth.SLICE_DZ, w.voltage_kv, w.calib,
                                 batch=args.batch, tune=tune, lanes=args.lanes)
        out_d = graphed.out
        ws, ws_bytes, prm = graphed.ws, graphed.ws_bytes, graphed.prm  # the steady-pass timing reuses them

        def step():  # noqa: F811
            graphed.replay()

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local_rank])

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(_physical_gpu(local_rank))
    starts, ends = _events(torch, args.steps), _events(torch, args.steps)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.ptyro_launch_count()
    for k in range(args.steps):
        flush.zero_()  # evict L2 between steps (256 MB > 126 MB L2)
        starts[k].record(stream)
        step()
        ends[k].record(stream)
    launches = lib.ptyro_launch_count() - launches0
    if graphed is not None:  # graph replays bypass the host-side launch counter
        launches = graphed.launches_per_replay * args.steps
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    updates = float(P) * S * args.steps * world
    value = updates / (total_ms * 1e-3)

    # sanity: every pattern sums to the aperture pixel count
    n_ap = float(((_aperture_mask(w)).sum()))
    sums = out_d.sum(dim=(1, 2))
    max_sum_err = float(((sums - n_ap).abs().max() / n_ap).item())

    # ---- dominant kernel: the steady-state pass over one batch of every lane, the lanes'
    # launches running side by side as in the captured forward
    reps = 20
    pass_ms = []
    parts = graphed.parts if graphed is not None else [(0, P, prm, ws, ws_bytes)]
    lane_streams = graphed.streams if (graphed is not None and graphed.streams) else [stream]
    for axis in (0, 1):
        s, e = _events(torch, 2)
        flush.zero_()
        s.record(stream)
        for (_, _, prm_i, ws_i, nbytes_i), st_i in zip(parts, lane_streams):
            st_i.wait_event(s)
            _lib.check(lib.ptyro_ms_steady_pass(ctypes.byref(prm_i), axis, reps, ws_i.data_ptr(), nbytes_i,
                                                st_i.cuda_stream))
        for st_i in lane_streams:
            stream.wait_stream(st_i)
        e.record(stream)
        torch.cuda.synchronize()
        pass_ms.append(s.elapsed_time(e) / reps)
    batch = sum(_batch_of(lib, prm_i, n) for (_, _, prm_i, _, _) in parts)
    avg_pass_s = statistics.mean(pass_ms) * 1e-3
    flops_per_launch = batch * synth.algorithmic_flops_per_update(n)
    achieved_tflops = flops_per_launch / avg_pass_s / 1e12
    peak = fp32_peak_tflops(torch, lib, dev)
    bytes_per_launch = batch * (2.0 * 8 * n * n) + 8.0 * n * n  # wave read+write, T read
    traffic = _ncu_traffic()

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        pot_h = torch.as_tensor(pot).pin_memory()
        modes_h = probe.cpu()[..., None].contiguous().pin_memory()
        pos_h = torch.as_tensor(pos, dtype=torch.float64).pin_memory()
        out_h = torch.empty((P, n, n), dtype=torch.float32).pin_memory()
        slices_obj = pb.PotentialSlices(pot_h, synth.SLICE_DZ, w.calib)
        beam_obj = pb.ProbeModes(modes_h, torch.ones(1, dtype=torch.float32).pin_memory(), w.calib)
        det_obj = pb.DetectorConfig(w.calib, w.calib * 100, 0.0, 0.0, pos_h, None, None)

        def e2e_step():  # the patterns stream to pinned host memory while later probes compute
            pb.stem_4d(slices_obj, beam_obj, mic, det_obj, out=out_h)

        e2e_step()
        torch.cuda.synchronize()
        k2 = max(1, min(args.steps, 5))
        barrier()
        torch.cuda.synchronize()
        s, e = _events(torch, 2)
        s.record(stream)
        for _ in range(k2):
            e2e_step()
        e.record(stream)
        torch.cuda.synchronize()
        e2e_ms = s.elapsed_time(e)
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        h2d = pot_h.numel() * 4 + modes_h.numel() * 8 + pos_h.numel() * 8 + 4
        e2e = {"value": float(P) * S * k2 * world / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(P * n * n * 4), "steps": k2}

    # the plain per-position path (one kernel per stage, one probe at a time) on a sample
    plain_probes = 8
    out_p = torch.empty((plain_probes, n, n), dtype=torch.float32, device=dev)
    pp = ms_params(n, S, 1, plain_probes, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, slices_d.stride(),
                   modes_d.stride())
    pws_b = lib.ptyro_ms_workspace_bytes(ctypes.byref(pp))
    pws = torch.empty(pws_b, dtype=torch.uint8, device=dev)

    def plain_step():
        _lib.check(lib.ptyro_ms_forward_plain(ctypes.byref(pp), slices_d.data_ptr(), modes_d.data_ptr(),
                                              weights_d.data_ptr(), pos_d.data_ptr(), out_p.data_ptr(),
                                              pws.data_ptr(), pws_b, stream.cuda_stream))

    plain_step()
    torch.cuda.synchronize()
    s, e = _events(torch, 2)
    s.record(stream)
    for _ in range(3):
        plain_step()
    e.record(stream)
    torch.cuda.synchronize()
    plain_value = 3.0 * plain_probes * S / (s.elapsed_time(e) * 1e-3)
    del pws

    cpu_baseline = None
    parity = None
    if cpu is not None:
        upd, wall = 0, 0.0
        while wall < args.cpu_seconds:
            u, t = cpu.step(1)
            upd += u
            wall += t
        # parity of the timed forward's patterns on a sample of probes (first, middle, last)
        idx = [0, P // 2, P - 1]
        want32, want64 = cpu.check(idx)
        got = out_d[idx].double().cpu().numpy()

        def rel(a, b):
            return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

        parity = {"probes": idx, "rel_l2_vs_float32_restatement": rel(got, want32),
                  "rel_l2_vs_float64_oracle": rel(got, want64),
                  "float32_restatement_vs_float64_oracle": rel(want32, want64)}
        cpu.close()
        cpu_baseline = {"value": upd / wall, "unit": UNIT, "cores": cpu.procs, "kind": "port",
                        "sample": f"{upd // S} probes of this workload (all 50 slices each), NumPy complex128 "
                                  f"oracle, one process per core"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "grid": n, "slices": S, "probes_per_gpu": P, "modes": 1,
                       "batch": _batch_of(lib, parts[0][2], n), "tune": tune, "cuda_graph": bool(args.graph),
                       "lanes": args.lanes if args.graph else 1, "voltage_kv": w.voltage_kv, "aperture_mrad": w.aperture_mrad,
                       "defocus_ang": w.defocus_ang, "c3_ang": w.c3_ang,
                       "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"dp{world} (probe shards, no collective)"},
            "roofline": {"bound": "fp32", "achieved": achieved_tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved_tflops / peak, "traffic": traffic,
                         "kernel": ("ms_pass_pair_kernel<16,16> steady-state pass (two lines per thread, f32x2; conv, x T, conv"
                                    + ("; column blocks by TMA)" if tune & 2048 else ")") if tune & 16 else "ms_pass_kernel<16,16> steady-state pass (conv, x T, conv)"),
                         "flops_per_launch": flops_per_launch, "launch_ms": [round(x, 4) for x in pass_ms],
                         "launch": f"one steady pass (row, column) of every lane side by side: {len(parts)} lanes, "
                                   f"{batch} wave slots in all",
                         "peak_source": "measured FP32 FMA stream (ptyro_fp32_fma_probe) in this run",
                         "hbm_achieved_gbs": bytes_per_launch / avg_pass_s / 1e9,
                         "hbm_algorithmic_bytes_per_launch": bytes_per_launch},
            "e2e": e2e,
            "plain_per_position": {"value": plain_value, "unit": UNIT, "probes_sampled": plain_probes,
                                   "fused_over_plain": value / plain_value},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu_baseline,
            "checks": {"pattern_sum_max_rel_err": max_sum_err,
                       "tma_wait_timeouts": int(lib.ptyro_pass_wait_timeouts()),
                       "device_status": graphed.status() if graphed is not None else None,
                       "sampled_parity": parity},
        }
        if world == 1 and not args.no_extras:
            # the other two halves of the metric, on the same GPU after the headline
            g = run_grad(argparse.Namespace(**{**vars(args), "steps": 12, "warmup": 3}), rank, world, local_rank)
            line["adjoint_over_forward"] = g["adjoint_over_forward"]
            line["gradient"] = {k: g[k] for k in ("metric", "value", "unit", "forward_ms",
                                                  "forward_with_residuals_ms", "adjoint_ms",
                                                  "adjoint_over_forward", "value_and_grad_over_forward",
                                                  "sparse_checkpoints", "config")}
            sv = run_serve(argparse.Namespace(**{**vars(args), "requests": 48}), rank, world, local_rank)
            line["p50_ms"], line["p99_ms"] = sv["p50_ms"], sv["p99_ms"]
            line["serving"] = {k: sv[k] for k in ("metric", "value", "unit", "p50_ms", "p99_ms", "mean_ms",
                                                  "requests", "completed", "makespan_s", "config", "batch_plan")}
        print(json.dumps(line), flush=True)


def _physical_gpu(local_rank: int) -> str:
    """nvidia-smi id of this rank's GPU (CUDA_VISIBLE_DEVICES entry if set)."""
    vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    return vis[local_rank] if local_rank < len(vis) else str(local_rank)


def _aperture_mask(w):
    from ptyrodactyl_b200.simulations import relativistic_wavelength_ang
    lam = relativistic_wavelength_ang(w.voltage_kv)
    fov = w.n * 0.01 * (w.calib * 100.0)
    f = np.fft.fftfreq(w.n) * w.n / fov
    q = np.sqrt(f[:, None] ** 2 + f[None, :] ** 2)
    return q <= (w.aperture_mrad / 1000.0) / lam


def _batch_of(lib, prm, n) -> int:
    if prm.batch > 0:
        return min(prm.batch, prm.num_probes)
    return max(1, min(prm.num_probes, (64 << 20) // (8 * n * n * prm.num_modes)))


def _ncu_traffic():
    """DRAM bytes per launch of the pass kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "pass_256_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


# ----------------------------------------------------------------------------- gradient leg
def run_grad(args, rank, world, local_rank):
    """Ptychographic gradient at the 256^2-window / 512^2-field workload: time the plain
    forward, the residual-recording forward and the adjoint; one JSON line."""
    import torch
    import ptyrodactyl_b200 as pb
    from ptyrodactyl_b200 import _lib
    from ptyrodactyl_b200.simulations import ms_params
    from ptyrodactyl_b200.recon import amplitude_loss

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    w = synth.CONFIG4
    n, S, P, F = w.n, w.num_slices, w.num_probes, w.field_n
    P = min(P, args.probes) if args.probes else P  # --probes: the first P scan windows (profiling cases)
    win = torch.as_tensor(w.windows()[:P], device=dev).contiguous()
    pos = torch.zeros((P, 2), dtype=torch.float64, device=dev)
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, w.defocus_ang, w.c3_ang, probe_shape=(n, n))
    probe = pb.make_probe(mic, pb.create_detector_config(w.calib))[..., None].contiguous()
    wts = torch.ones(1, dtype=torch.float32, device=dev)
    truth = torch.as_tensor(w.field(0), device=dev)
    model = torch.as_tensor(w.field(1), device=dev)  # another frozen-phonon draw: the current estimate
    clean = pb.run_forward(truth, synth.SLICE_DZ, probe, wts, pos, w.voltage_kv, w.calib, w.calib, windows=win)
    rng = np.random.default_rng(w.seed)
    targets = torch.as_tensor(synth.poisson_targets(clean.cpu().numpy().astype(np.float64), w.dose, rng),
                              dtype=torch.float32, device=dev)
    from ptyrodactyl_b200.autodiff import _ckpt_for, run_backward, run_forward_ckpt
    k = _ckpt_for(S, args.ckpt, n, P)  # the library's default: every slice when the residuals fit
    prm = ms_params(n, S, 1, P, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, model.stride(), probe.stride(),
                    0, default_tune(n) if args.tune < 0 else args.tune, F, win)
    bprm = ms_params(n, S, 1, P, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, model.stride(), probe.stride(),
                     args.bwd_batch, prm.tune, F, win)
    res = torch.empty(lib.ptyro_ms_residual_bytes(ctypes.byref(prm), k) // 4, dtype=torch.float32, device=dev)
    out = torch.empty((P, n, n), dtype=torch.float32, device=dev)
    g_field = torch.empty_like(model)
    g_modes = torch.empty_like(probe)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def fwd():  # the library's forward (concurrent probe lanes, as stem_4d runs it)
        pb.run_forward(model, synth.SLICE_DZ, probe, wts, pos, w.voltage_kv, w.calib, w.calib, out=out,
                       tune=prm.tune, windows=win)

    def fwd_ckpt():  # the library's residual-recording forward (concurrent probe lanes, as stem_4d records)
        run_forward_ckpt(model, probe, wts, pos, k, synth.SLICE_DZ, w.voltage_kv, w.calib, w.calib, 0, prm.tune, win,
                         out, res)

    gbuf = {}

    def loss_grad():
        o = out.detach().requires_grad_(True)
        loss = amplitude_loss(o, targets)
        loss.backward()
        gbuf["g"] = o.grad.contiguous()
        gbuf["loss"] = loss.detach()

    def bwd():  # the library's adjoint (concurrent probe lanes, as stem_4d's backward runs it)
        run_backward(model, probe, wts, pos, res, gbuf["g"], k, synth.SLICE_DZ, w.voltage_kv, w.calib, w.calib,
                     args.bwd_batch, prm.tune, win, g_field, g_modes)
        if world > 1:  # each rank holds its probes' share of dL/dV: one NCCL all-reduce sums them
            import torch.distributed as dist
            dist.all_reduce(g_field)

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            flush.zero_()
            s, e = _events(torch, 2)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e))
        return statistics.median(ts)

    for _ in range(args.warmup):
        fwd(); fwd_ckpt(); loss_grad(); bwd()
    torch.cuda.synchronize()
    reps = max(3, args.steps // 4)
    t_f = timed(fwd, reps)
    t_fc = timed(fwd_ckpt, reps)
    loss_grad()
    t_b = timed(bwd, reps)
    # the sparser checkpoints (ceil(sqrt(S)), far less residual memory) with the lockstep
    # adjoint that rebuilds the forward wave between them
    t_b_sparse, k_sparse = None, int(np.ceil(np.sqrt(S)))
    if k == 1 and k_sparse > 1 and world == 1:
        k_main = k
        k = k_sparse
        res_main = res
        res = torch.empty(lib.ptyro_ms_residual_bytes(ctypes.byref(prm), k) // 4, dtype=torch.float32, device=dev)
        fwd_ckpt()
        loss_grad()
        bwd()
        torch.cuda.synchronize()
        t_b_sparse = timed(bwd, reps)
        k, res = k_main, res_main
    if world > 1:  # whole-job times: the slowest rank
        import torch.distributed as dist
        tt = torch.tensor([t_f, t_fc, t_b], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_f, t_fc, t_b = (float(v) for v in tt.tolist())
    updates = float(P) * S * world
    line = {
        "metric": "ptychographic gradient: value+grad probe-slice updates/s (256^2 windows, 512^2 field)",
        "value": updates / ((t_fc + t_b) * 1e-3), "unit": UNIT, "n_gpus": world, "mode": "grad",
        "forward_ms": t_f, "forward_with_residuals_ms": t_fc, "adjoint_ms": t_b,
        "adjoint_over_forward": t_b / t_f, "value_and_grad_over_forward": (t_fc + t_b) / t_f,
        "sparse_checkpoints": None if t_b_sparse is None else {
            "ckpt_every": k_sparse, "adjoint_ms": t_b_sparse, "adjoint_over_forward": t_b_sparse / t_f,
            "residual_bytes": int(lib.ptyro_ms_residual_bytes(ctypes.byref(prm), k_sparse))},
        "loss": float(gbuf["loss"]), "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "grid": n, "field": F, "slices": S, "probes": P, "ckpt_every": k,
                   "residual_bytes": int(res.numel() * 4), "backward_batch": bprm.batch,
                   "lanes": "forward, recording forward and adjoint as the library runs them: two concurrent "
                            "probe lanes",
                   "targets": f"Poisson noise at {w.dose:g} e- per pattern", "loss": "amplitude"},
    }
    del res
    return line


# ----------------------------------------------------------------------------- 512^2 leg
def run_config3(args, rank, world, local_rank):
    """512^2 grid, 32x32 cell, 100 slices, frozen-phonon average of 4 configurations,
    on the 128x128 scan (or a sample of ``--probes`` positions); one JSON line."""
    import torch
    import ptyrodactyl_b200 as pb
    from ptyrodactyl_b200 import _lib

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = synth.CONFIG3
    n, S = w.n, w.num_slices
    pos_all = synth.raster_positions(w)
    probes = args.probes or pos_all.shape[0]  # default: the full 128x128 scan
    idx = np.linspace(0, pos_all.shape[0] - 1, probes).astype(np.int64)
    pos = torch.as_tensor(pos_all[idx], device=dev).contiguous()
    pots = [torch.as_tensor(synth.potential_slices(w, phonon=k), device=dev) for k in range(w.phonon_configs)]
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, probe_shape=(n, n))
    modes = pb.make_probe(mic, pb.create_detector_config(w.calib))[..., None].contiguous()
    wq = torch.full((1,), 1.0 / len(pots), dtype=torch.float32, device=dev)
    out = torch.zeros((probes, n, n), dtype=torch.float32, device=dev)

    def step():
        out.zero_()
        for v in pots:
            pb.run_forward(v, synth.SLICE_DZ, modes, wq, pos, w.voltage_kv, w.calib, w.calib, out=out,
                           accumulate=True, batch=args.batch, tune=None if args.tune < 0 else args.tune)

    for _ in range(max(1, args.warmup // 3)):
        step()
    torch.cuda.synchronize()
    s, e = _events(torch, 2)
    reps = max(1, args.steps // 10)
    s.record()
    for _ in range(reps):
        step()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    updates = float(probes) * S * len(pots)
    sums = out.sum(dim=(1, 2))
    n_ap = float(_aperture_mask(w).sum())
    line = {"metric": "probe-slice updates/s at 512^2 (100 slices, 4 frozen-phonon configurations averaged)",
            "mode": "config3", "value": updates / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "tflops_algorithmic": updates / (ms * 1e-3) * synth.algorithmic_flops_per_update(n) / 1e12,
            "n_gpus": world, "dtype": "f32", "data": "synthetic",
            "checks": {"pattern_sum_max_rel_err": float(((sums - n_ap).abs().max() / n_ap).item()),
                       "tma_wait_timeouts": int(_lib.load().ptyro_pass_wait_timeouts())},
            "config": {"workload": w.name, "grid": n, "slices": S, "probes_sampled": probes,
                       "probes_full_scan": w.num_probes, "phonon_configs": len(pots), "batch": args.batch,
                       "tune": default_tune(w.n) if args.tune < 0 else args.tune}}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- 128^2 leg
def run_config1(args, rank, world, local_rank):
    """128^2 grid, 8x8 cell, 20 slices: the pass engine (wave slots through L2 once per
    slice) against the wave-resident kernel (tune bit 32768: one CTA per probe, the
    wave in shared memory across all slices), both replayed from CUDA graphs, on the
    16x16 scan (256 probes) and on a 8192-probe sample (the scan at 32 sub-pixel
    offsets) that fills the GPU; one JSON line."""
    import torch
    import ptyrodactyl_b200 as pb
    from ptyrodactyl_b200.graphs import GraphedForward

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = synth.CONFIG1
    n, S = w.n, w.num_slices
    slices = torch.as_tensor(synth.potential_slices(w), device=dev)
    mic = pb.create_microscope_config(w.voltage_kv, w.aperture_mrad, probe_shape=(n, n))
    modes = pb.make_probe(mic, pb.create_detector_config(w.calib))[..., None].contiguous()
    wts = torch.ones(1, dtype=torch.float32, device=dev)
    scan = synth.raster_positions(w)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    base = default_tune(n) if args.tune < 0 else args.tune
    result = {}
    for label, reps_pos in (("scan_256", 1), ("sample_8192", 32)):
        pos = np.concatenate([scan + 0.031 * i for i in range(reps_pos)])
        pos_d = torch.as_tensor(pos, device=dev).contiguous()
        P = pos.shape[0]
        row = {"probes": P}
        outs = {}
        for kind, tune in (("pass_engine", base & ~32768), ("resident", base | 32768)):
            g = GraphedForward(slices, modes, wts, pos_d, synth.SLICE_DZ, w.voltage_kv, w.calib, tune=tune,
                               batch=P if kind == "resident" else 0)
            for _ in range(args.warmup):
                g.replay()
            torch.cuda.synchronize()
            reps = max(5, args.steps)
            ts = []
            for _ in range(reps):
                flush.zero_()
                s_, e_ = _events(torch, 2)
                s_.record()
                g.replay()
                e_.record()
                torch.cuda.synchronize()
                ts.append(s_.elapsed_time(e_))
            g.check()
            ms = statistics.median(ts)
            upd = float(P) * S / (ms * 1e-3)
            row[kind] = {"ms_per_forward": ms, "updates_per_s": upd,
                         "tflops_algorithmic": upd * synth.algorithmic_flops_per_update(n) / 1e12,
                         "launches_per_forward": g.launches_per_replay, "tune": tune}
            outs[kind] = g.out.clone()
        row["bit_identical"] = bool(torch.equal(outs["pass_engine"], outs["resident"]))
        row["resident_over_pass_engine"] = row["resident"]["updates_per_s"] / row["pass_engine"]["updates_per_s"]
        result[label] = row
    line = {"metric": "probe-slice updates/s at 128^2 (20 slices): pass engine vs wave-resident kernel",
            "mode": "config1", "unit": UNIT, "n_gpus": world, "dtype": "f32", "data": "synthetic",
            "value": max(result["sample_8192"]["pass_engine"]["updates_per_s"],
                         result["sample_8192"]["resident"]["updates_per_s"]),
            "results": result,
            "config": {"workload": w.name, "grid": n, "slices": S, "voltage_kv": w.voltage_kv,
                       "aperture_mrad": w.aperture_mrad, "l2": "flushed (256 MB write) before every timed forward"}}
    return line


# ----------------------------------------------------------------------------- serving leg
def run_serve(args, rank, world, local_rank):
    """Poisson-arrival mix of simulations and gradient solves through the server;
    p50/p99 latency and aggregate probe-slice updates/s (one JSON line)."""
    import torch
    from ptyrodactyl_b200.serving import Request, Server, serving_mix

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    srv = Server(arena_bytes=int(args.arena_gb * (1 << 30)), max_slots=args.max_slots, device=dev)
    smax = 100
    for n in (64, 128, 256, 512):
        w = synth.Workload(f"serve-{n}", n, n * 4 // 64 if n >= 64 else 1, smax, (1, 1), 200.0, 20.0, seed=5)
        srv.add_potential(f"p{n}", synth.potential_slices(w))
    calib = 4 * synth.LATTICE_A / 64  # 4 cells per 64 px at every edge

    def build(spec, arrival_abs):
        n, p = spec["n"], spec["num_probes"]
        side = int(np.ceil(np.sqrt(p)))
        fov = n * calib
        g = (np.arange(side) - (side - 1) / 2.0) * (fov / side)
        yy, xx = np.meshgrid(g, g, indexing="ij")
        pos = np.stack([yy.ravel(), xx.ravel()], axis=1)[:p]
        req = Request(n=n, num_slices=spec["num_slices"], positions=pos, voltage_kv=spec["voltage_kv"],
                      aperture_mrad=spec["aperture_mrad"], defocus_ang=spec["defocus_ang"], kind=spec["kind"],
                      potential_key=f"p{n}", calib_ang=calib, arrival_s=arrival_abs)
        if spec["kind"] == "grad":
            gen = torch.Generator(device=dev)
            gen.manual_seed(spec["seed"])
            req.targets = torch.rand((p, n, n), generator=gen, device=dev) * (2.0 / (n * n))
        return req

    # warm-up: one request of every grid edge and kind (module loading, first launches)
    for n in (64, 128, 256, 512):
        for kind in ("forward", "grad"):
            srv.submit(build(dict(n=n, num_probes=4, num_slices=5, voltage_kv=200.0, aperture_mrad=20.0,
                                  defocus_ang=0.0, kind=kind, seed=1), time.perf_counter()))
    srv.drain()
    srv.finished.clear()
    mix = serving_mix(args.requests, args.seed, args.rate)

    def play():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        i = 0
        while i < len(mix) or srv.active:
            now = time.perf_counter() - t0
            while i < len(mix) and mix[i]["arrival_s"] <= now:
                srv.submit(build(mix[i], t0 + mix[i]["arrival_s"]))
                i += 1
            if srv.active:
                srv.poll()
            elif i < len(mix):
                time.sleep(max(0.0, min(0.001, mix[i]["arrival_s"] - now)))
        torch.cuda.synchronize()
        return t0, time.perf_counter()

    # an untimed rehearsal of the same mix first: the first pass over a fresh device
    # pays one-time costs (first touches of arena pages, first launches of each
    # request shape) that a long-running server has behind it
    play()
    srv.finished.clear()
    t0, t_end = play()
    lat = np.array([r.latency_s for r in srv.finished]) * 1e3
    upd = sum(r.request.updates for r in srv.finished)
    ok = sum(1 for r in srv.finished if r.state == 2)
    plan = {"probes_64": run_plan_leg(srv, build, mix, dev, max_probes=64),
            "probes_4": run_plan_leg(srv, build, mix, dev, max_probes=4)}
    srv.close()
    line = {
        "metric": "serving mix: p50/p99 latency and aggregate probe-slice updates/s", "mode": "serve",
        "value": upd / (t_end - t0), "unit": UNIT, "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "requests": len(mix),
        "completed": ok, "makespan_s": t_end - t0, "n_gpus": world, "dtype": "f32", "data": "synthetic",
        "config": {"grids": [64, 128, 256, 512], "slices": "5-100 log-uniform", "probes": "1-4096 log-uniform",
                   "kv": "60-300", "aperture_mrad": "10-30", "grad_fraction": 0.3, "rate_hz": args.rate,
                   "seed": args.seed, "arena_gb": args.arena_gb, "max_slots": args.max_slots,
                   "admission": "HBM footprint (arena) + wave-slot budget",
                   "targets": "uniform random patterns (gradient cost does not depend on them)"},
        "batch_plan": plan,
    }
    return line


def run_plan_leg(srv, build, mix, dev, jobs=16, max_probes=64, reps=3):
    """A fixed batch of uneven requests (the first ``jobs`` of the serving mix, each
    cut to at most ``max_probes`` probes, so the batch is launch-bound like small
    serving traffic) run twice: through the stepped scheduler (host ticks, staging
    copies, events; wall time) and as one CUDA-graph replay of the same jobs recorded
    as a batch plan (``ptyro_plan_*``; device time and wall time). The replay's
    results are checked bit for bit against the scheduler's."""
    import torch
    from ptyrodactyl_b200 import _lib

    lib = _lib.load()
    specs = [dict(m, num_probes=min(m["num_probes"], max_probes)) for m in mix[:jobs]]
    reqs = [build(sp, 0.0) for sp in specs]
    updates = sum(r.updates for r in reqs)

    def scheduled():
        srv.finished.clear()
        for r in reqs:
            srv.submit(r)
        srv.drain()
        return {id(res.request): res for res in srv.finished}

    scheduled()  # warm-up
    walls = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        want = scheduled()
        torch.cuda.synchronize()
        walls.append(time.perf_counter() - t)
    plan, results = srv.plan(reqs)
    before = lib.ptyro_launch_count()
    plan.launch()
    torch.cuda.synchronize()
    launches = int(lib.ptyro_launch_count() - before)
    plan.capture()
    plan.replay()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev_ms, plan_walls = [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        s.record()
        plan.replay()
        e.record()
        torch.cuda.synchronize()
        plan_walls.append(time.perf_counter() - t)
        dev_ms.append(s.elapsed_time(e))
    identical = all(torch.equal(res.patterns, want[id(r)].patterns) for r, res in zip(reqs, results))
    status = plan.status()
    plan.close()
    sched_s, plan_s = float(np.median(walls)), float(np.median(plan_walls))
    return {"jobs": len(reqs), "grad_jobs": sum(1 for r in reqs if r.kind == "grad"),
            "grids": sorted({r.n for r in reqs}), "probes_per_job_max": max_probes, "updates": updates,
            "scheduler_wall_ms": sched_s * 1e3, "plan_replay_wall_ms": plan_s * 1e3,
            "plan_replay_device_ms": float(np.median(dev_ms)), "replay_over_scheduler": sched_s / plan_s,
            "plan_updates_per_s": updates / plan_s, "kernel_launches_per_replay": launches,
            "bit_identical_to_scheduler": bool(identical), "device_status": int(status)}


# ----------------------------------------------------------------------------- profiling case
def run_profile_case(args, rank, world, local_rank):
    """A small, self-checking case of the forward engine for profilers: one batched
    forward over ``--probes`` scan positions of the perovskite workload (``--grid``
    edge, ``--slices`` slices, one batch), then ``--reps`` steady-state passes per axis
    (``ptyro_ms_steady_pass``) on the wave slots the forward left in the workspace.
    Pass-kernel launches: slices + 4 in the forward (setup kernels aside; one for the
    wave-resident kernel, tune bit 32768), then ``--reps`` row
    passes and ``--reps`` column passes. Exits non-zero if the patterns are not finite
    or the device status word is set."""
    import torch
    from ptyrodactyl_b200 import _lib
    from ptyrodactyl_b200.simulations import make_probe, ms_params
    from ptyrodactyl_b200.types import create_detector_config, create_microscope_config

    n, probes, reps, S = args.grid, args.probes or 2048, args.reps, args.slices
    tune = default_tune(n) if args.tune < 0 else args.tune
    w = synth.CONFIG2
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    if n == w.n:
        pot = torch.as_tensor(synth.potential_slices(w, num_slices=S), device=dev)
    else:
        pot = torch.rand((n, n, S), generator=torch.Generator(device=dev).manual_seed(1), device=dev) * 50
    mic = create_microscope_config(w.voltage_kv, w.aperture_mrad, probe_shape=(n, n))
    probe = make_probe(mic, create_detector_config(w.calib))[..., None].contiguous()
    pos = torch.as_tensor(synth.raster_positions(w), device=dev)[:probes].contiguous()
    probes = pos.shape[0]
    wt = torch.ones(1, device=dev)
    prm = ms_params(n, S, 1, probes, w.voltage_kv, synth.SLICE_DZ, w.calib, w.calib, pot.stride(), probe.stride(),
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
    status = int(ws[:4].view(torch.int32).item())
    print(f"profile case n={n} probes={probes} reps={reps} tune={tune}: pattern sum {total:.6g}, status {status}")
    return 0 if (total == total and abs(total) != float("inf") and status == 0) else 1


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return
    procs = min(_host_cores(), 64)
    cpu = CpuOracle(procs)
    for _ in range(args.warmup):
        cpu.step(1)
    upd, wall = 0, 0.0
    for _ in range(args.steps):
        u, t = cpu.step(1)
        upd += u
        wall += t
    cpu.close()
    value = upd / wall
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD.name, "grid": WORKLOAD.n, "slices": WORKLOAD.num_slices,
                   "probes": WORKLOAD.num_probes, "sample_probes_per_step": procs},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"{procs} probes (all 50 slices) per step, NumPy complex128 restatement of "
                                   "the reference's x64 stem_4d (JAX is not installed), one process per core"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--tune", type=int, default=-1,
                    help="pass-kernel variant bits; -1: the measured default for the grid edge")
    ap.add_argument("--graph", type=int, default=1, help="1: time CUDA-graph replays of the captured forward")
    ap.add_argument("--lanes", type=int, default=2, help="concurrent probe ranges (streams) in the captured forward")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="forward mode: skip the gradient and serving legs that follow the headline")
    ap.add_argument("--mode", choices=("forward", "grad", "serve", "config1", "config3", "profile-case"),
                    default="forward")
    ap.add_argument("--probes", type=int, default=0,
                    help="config3 mode: scan positions sampled (0: the full 128x128 scan); profile-case mode: "
                         "probes in the one batch (0: 2048); grad mode: the first scan windows (0: all 1024)")
    ap.add_argument("--grid", type=int, default=256, help="profile-case mode: grid edge")
    ap.add_argument("--reps", type=int, default=1, help="profile-case mode: steady passes per axis")
    ap.add_argument("--slices", type=int, default=2, help="profile-case mode: slices of the forward")
    ap.add_argument("--requests", type=int, default=64, help="serve mode: requests in the mix")
    ap.add_argument("--rate", type=float, default=20.0, help="serve mode: Poisson arrival rate (1/s)")
    ap.add_argument("--seed", type=int, default=5, help="serve mode: mix seed")
    ap.add_argument("--arena-gb", type=float, default=48.0, help="serve mode: scheduler arena")
    ap.add_argument("--max-slots", type=int, default=1024, help="serve mode: wave slots in flight")
    ap.add_argument("--ckpt", type=int, default=0, help="gradient mode: checkpoint spacing (0 = sqrt(S))")
    ap.add_argument("--bwd-batch", type=int, default=0, help="gradient mode: probes per adjoint batch")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else max(args.warmup, 1)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.mode in ("grad", "serve", "config1"):
            line = {"grad": run_grad, "serve": run_serve, "config1": run_config1}[args.mode](args, rank, world,
                                                                                      local_rank)
            if rank == 0:
                print(json.dumps(line), flush=True)
        elif args.mode == "config3":
            run_config3(args, rank, world, local_rank)
        elif args.mode == "profile-case":
            sys.exit(run_profile_case(args, rank, world, local_rank))
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
