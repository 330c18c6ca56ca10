"""Serving: continuous batching of multislice simulations and gradient solves.

:class:`Scheduler` wraps the native multi-job scheduler (``ptyro_sched_*``): jobs of
any grid edge, slice count and scan size are admitted as arena memory and wave
slots free up, and every tick advances all running jobs by one pass in shared
multi-job launches. :class:`Server` adds the request side: device-resident
potential and probe caches, per-request output buffers, arrival handling and
latency bookkeeping (p50/p99 and aggregate probe-slice updates/s).

The reference has no serving layer (it runs one jitted ``stem_4d`` call at a
time); this module exists for the serving pattern of the B200 build.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .simulations import default_tune, make_probe, ms_params, relativistic_wavelength_ang
from .types import create_detector_config, create_microscope_config


class Scheduler:
    """Owner of one native scheduler and its device arena (allocated once)."""

    def __init__(self, arena_bytes: int, max_slots: int = 1024, device: Optional[torch.device] = None):
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        self.arena = torch.empty(int(arena_bytes), dtype=torch.uint8, device=self.device)
        handle = ctypes.c_void_p()
        _lib.check(self.lib.ptyro_sched_create(self.device.index or 0, self.arena.data_ptr(), int(arena_bytes),
                                               int(max_slots), ctypes.byref(handle)))
        self.handle = handle
        self._keep: Dict[int, tuple] = {}  # job id -> buffers kept alive until the job is released

    def job_bytes(self, desc: _lib.JobDesc) -> int:
        return int(self.lib.ptyro_sched_job_bytes(ctypes.byref(desc)))

    def submit(self, desc: _lib.JobDesc, keep: tuple = ()) -> int:
        jid = ctypes.c_int64()
        _lib.check(self.lib.ptyro_sched_submit(self.handle, ctypes.byref(desc), ctypes.byref(jid)))
        self._keep[jid.value] = (desc,) + tuple(keep)
        return jid.value

    def step(self) -> Tuple[int, int]:
        running, queued = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self.lib.ptyro_sched_step(self.handle, ctypes.byref(running), ctypes.byref(queued)))
        return running.value, queued.value

    def state(self, jid: int) -> int:
        st = ctypes.c_int32()
        _lib.check(self.lib.ptyro_sched_job_state(self.handle, jid, ctypes.byref(st)))
        return st.value

    def cancel(self, jid: int) -> None:
        _lib.check(self.lib.ptyro_sched_cancel(self.handle, jid))

    def release(self, jid: int) -> None:
        _lib.check(self.lib.ptyro_sched_release(self.handle, jid))
        self._keep.pop(jid, None)

    def memory(self) -> Tuple[int, int]:
        fb, fs = ctypes.c_size_t(), ctypes.c_int32()
        _lib.check(self.lib.ptyro_sched_memory(self.handle, ctypes.byref(fb), ctypes.byref(fs)))
        return fb.value, fs.value

    def run(self, jids: List[int], timeout_s: float = 600.0) -> None:
        """Step until every job in ``jids`` has left the scheduler."""
        t0 = time.time()
        pending = set(jids)
        while pending:
            self.step()
            pending = {j for j in pending if self.state(j) in (_lib.JOB_QUEUED, _lib.JOB_RUNNING)}
            if time.time() - t0 > timeout_s:
                raise TimeoutError(f"{len(pending)} jobs still running after {timeout_s} s")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.ptyro_sched_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """A fixed batch of jobs (uneven grid edges, slice counts and scan sizes, forward
    and gradient) recorded once as the scheduler would run them (``ptyro_plan_*``):
    every tick one multi-job launch per pass kind, all descriptors in device memory.
    :meth:`launch` enqueues the whole batch on the current stream with no host
    synchronisation; :meth:`capture` records that into a CUDA graph and
    :meth:`replay` reruns every job on the current contents of its input buffers.
    Inputs must be ready on the launching stream; the arena holds all jobs' scratch."""

    def __init__(self, descs: List[_lib.JobDesc], keep: tuple = (), device=None):
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._descs = (_lib.JobDesc * len(descs))(*descs)
        self.num_jobs = len(descs)
        nbytes = int(self.lib.ptyro_plan_bytes(self._descs, self.num_jobs))
        if nbytes == 0:
            _lib.check(_lib.PTYRO_ERR_INVALID)
        self.arena = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ptyro_plan_create(self.device.index or 0, self._descs, self.num_jobs,
                                                  self.arena.data_ptr(), nbytes, ctypes.byref(handle)))
        self.handle = handle
        self._keep = keep
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def launch(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ptyro_plan_launch(self.handle, st.cuda_stream))

    def capture(self) -> torch.cuda.CUDAGraph:
        """Record one launch into a CUDA graph (after one plain launch, which sets the
        kernels' per-device attributes outside the capture)."""
        main = torch.cuda.current_stream(self.device)
        self.launch(main)
        side = torch.cuda.Stream(device=self.device)
        side.wait_stream(main)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self.launch(side)
        main.wait_stream(side)
        self.graph = g
        return g

    def replay(self) -> None:
        if self.graph is None:
            raise RuntimeError("capture() the plan first")
        self.graph.replay()

    def status(self) -> int:
        """OR of the jobs' device status words after the last launch (synchronises)."""
        base = self.arena.data_ptr()
        word = 0
        for i in range(self.num_jobs):
            ptr = ctypes.c_void_p()
            _lib.check(self.lib.ptyro_plan_job_status(self.handle, i, ctypes.byref(ptr)))
            off = int(ptr.value) - base
            word |= int(self.arena[off:off + 4].view(torch.int32).item())
        return word

    def check(self, what: str = "batch plan") -> None:
        word = self.status()
        if word:
            raise _lib.DeviceStatusError(f"{what}: device status {word:#x} (a bounded wait gave up)")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.graph = None
            self.lib.ptyro_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Request:
    """One simulation (kind "forward") or gradient solve (kind "grad")."""

    n: int
    num_slices: int
    positions: np.ndarray          # (P, 2) Angstrom shifts
    voltage_kv: float
    aperture_mrad: float
    defocus_ang: float = 0.0
    c3_ang: float = 0.0
    kind: str = "forward"
    potential_key: str = ""        # device-resident potential (F >= n, S >= num_slices)
    calib_ang: float = 0.2
    slice_thickness: float = 1.95
    arrival_s: float = 0.0
    targets: Optional[torch.Tensor] = None  # grad: (P, n, n) float32 on the device
    batch: int = 0

    @property
    def updates(self) -> int:
        return int(self.positions.shape[0]) * int(self.num_slices)


@dataclass
class Result:
    request: Request
    patterns: torch.Tensor
    grad_potential: Optional[torch.Tensor] = None
    grad_modes: Optional[torch.Tensor] = None
    loss: Optional[torch.Tensor] = None
    submit_s: float = 0.0
    done_s: float = 0.0
    state: int = _lib.JOB_QUEUED

    @property
    def latency_s(self) -> float:
        return self.done_s - self.request.arrival_s


class Server:
    """Request front end over :class:`Scheduler` with device-resident caches."""

    def __init__(self, arena_bytes: int = 16 << 30, max_slots: int = 1024, device=None):
        self.sched = Scheduler(arena_bytes, max_slots, device)
        self.device = self.sched.device
        self.potentials: Dict[str, torch.Tensor] = {}
        self.probes: Dict[tuple, torch.Tensor] = {}
        self.weights = torch.ones(1, dtype=torch.float32, device=self.device)
        self.active: Dict[int, Result] = {}
        self.finished: List[Result] = []

    # ---- caches
    def add_potential(self, key: str, slices) -> None:
        """Keep a potential (F, F, S) float32 on the device under ``key``."""
        t = torch.as_tensor(np.asarray(slices, np.float32) if not isinstance(slices, torch.Tensor) else slices,
                            dtype=torch.float32).to(self.device).contiguous()
        self.potentials[key] = t

    def probe(self, n: int, voltage_kv: float, aperture_mrad: float, calib_ang: float, defocus_ang: float,
              c3_ang: float) -> torch.Tensor:
        key = (n, round(voltage_kv, 6), round(aperture_mrad, 6), round(calib_ang, 9), round(defocus_ang, 6),
               round(c3_ang, 9))
        pr = self.probes.get(key)
        if pr is None:
            mic = create_microscope_config(voltage_kv, aperture_mrad, defocus_ang, c3_ang, probe_shape=(n, n))
            pr = make_probe(mic, create_detector_config(calib_ang))[..., None].contiguous()
            self.probes[key] = pr
        return pr

    # ---- requests
    def submit(self, req: Request) -> int:
        d, res, keep = self._job(req)
        # the inputs above were written on torch's stream; the scheduler's streams wait for them
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(self.device))
        d.ready_event = ready.cuda_event
        keep = keep + (ready,)
        res.submit_s = time.perf_counter()
        jid = self.sched.submit(d, keep)
        self.active[jid] = res
        return jid

    def plan(self, requests: List[Request]) -> Tuple["BatchPlan", List[Result]]:
        """The requests as one recorded :class:`BatchPlan` (not submitted to the
        scheduler) and their result buffers, filled by every launch or replay."""
        jobs = [self._job(r) for r in requests]
        plan = BatchPlan([d for d, _, _ in jobs], keep=tuple(k for _, _, k in jobs), device=self.device)
        return plan, [r for _, r, _ in jobs]

    def _job(self, req: Request) -> Tuple[_lib.JobDesc, Result, tuple]:
        pot = self.potentials[req.potential_key]
        if pot.shape[0] != req.n or pot.shape[1] != req.n or pot.shape[2] < req.num_slices:
            raise ValueError("the cached potential must be (n, n, S_max) with S_max >= the request's slices")
        slices = pot[:, :, :req.num_slices]  # view of the resident cache: no copy
        modes = self.probe(req.n, req.voltage_kv, req.aperture_mrad, req.calib_ang, req.defocus_ang, req.c3_ang)
        P = int(req.positions.shape[0])
        pos = torch.as_tensor(np.asarray(req.positions, np.float64), device=self.device).reshape(P, 2).contiguous()
        out = torch.empty((P, req.n, req.n), dtype=torch.float32, device=self.device)
        d = _lib.JobDesc()
        # the per-edge launch variant also lays out the interleaved transmission tables
        # that the paired multi-job passes read
        d.p = ms_params(req.n, req.num_slices, 1, P, req.voltage_kv, req.slice_thickness, req.calib_ang,
                        req.calib_ang, slices.stride(), modes.stride(), req.batch, default_tune(req.n))
        d.kind = _lib.PTYRO_JOB_GRADIENT if req.kind == "grad" else _lib.PTYRO_JOB_FORWARD
        d.potential, d.modes, d.weights, d.positions = (slices.data_ptr(), modes.data_ptr(),
                                                        self.weights.data_ptr(), pos.data_ptr())
        d.patterns = out.data_ptr()
        res = Result(req, out)
        keep = (slices, modes, pos, out)
        if req.kind == "grad":
            if req.targets is None:
                raise ValueError("gradient requests need targets")
            tg = req.targets.to(self.device, torch.float32).contiguous()
            # dV is written with the potential's strides: a buffer shaped like the cache entry
            gbase = torch.empty_like(pot)
            res.grad_potential = gbase[:, :, :req.num_slices]
            res.grad_modes = torch.empty_like(modes)
            res.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
            d.targets = tg.data_ptr()
            d.grad_potential = res.grad_potential.data_ptr()
            d.grad_modes = res.grad_modes.data_ptr()
            d.loss = res.loss.data_ptr()
            keep = keep + (tg, gbase, res.grad_modes, res.loss)
        return d, res, keep

    def poll(self) -> int:
        """One scheduler tick; move finished jobs to :attr:`finished`. Returns jobs in flight."""
        self.sched.step()
        now = time.perf_counter()
        for jid in list(self.active):
            st = self.sched.state(jid)
            if st not in (_lib.JOB_QUEUED, _lib.JOB_RUNNING):
                res = self.active.pop(jid)
                res.state = st
                res.done_s = now
                self.finished.append(res)
                self.sched.release(jid)
        return len(self.active)

    def drain(self, timeout_s: float = 900.0) -> None:
        t0 = time.time()
        while self.active:
            self.poll()
            if time.time() - t0 > timeout_s:
                raise TimeoutError("server did not drain")

    def close(self) -> None:
        self.sched.close()


# ----------------------------------------------------------------------------- the serving mix
SERVE_GRIDS = (64, 128, 256, 512)


def serving_mix(num_requests: int, seed: int, rate_hz: float, grad_fraction: float = 0.3) -> List[dict]:
    """Seeded request stream: Poisson arrivals at ``rate_hz``; grid uniform over
    {64, 128, 256, 512}; slices 5-100 and scan 1-4096 positions log-uniform;
    60-300 kV, 10-30 mrad uniform; ``grad_fraction`` forward + adjoint solves."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(num_requests):
        t += rng.exponential(1.0 / rate_hz)
        n = int(rng.choice(SERVE_GRIDS))
        s = int(round(math.exp(rng.uniform(math.log(5), math.log(100)))))
        p = int(round(math.exp(rng.uniform(0.0, math.log(4096)))))
        out.append(dict(arrival_s=t, n=n, num_slices=s, num_probes=p, voltage_kv=float(rng.uniform(60, 300)),
                        aperture_mrad=float(rng.uniform(10, 30)), defocus_ang=float(rng.uniform(-80, 80)),
                        kind="grad" if rng.uniform() < grad_fraction else "forward", seed=int(rng.integers(1 << 30))))
    return out
