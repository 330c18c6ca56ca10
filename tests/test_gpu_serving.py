"""The multi-job scheduler and the server (GPU): every result equals the same job
run alone, forward and gradient jobs of different sizes share launches, admission
waits for memory, cancellation and rejection are handled on the host."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from ptyrodactyl_b200 import _lib, synth
from ptyrodactyl_b200.recon import amplitude_loss
from ptyrodactyl_b200.serving import Request, Server

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def server():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    srv = Server(arena_bytes=4 << 30, max_slots=512)
    rng = np.random.default_rng(0)
    for n in (64, 128, 256, 512):
        srv.add_potential(f"p{n}", rng.uniform(0.0, 40.0, (n, n, 24)).astype(np.float32))
    yield srv
    srv.close()


def _req(n, s, p, kind="forward", seed=0, kv=200.0, targets=None):
    rng = np.random.default_rng(seed)
    return Request(n=n, num_slices=s, positions=rng.uniform(-3, 3, (p, 2)), voltage_kv=kv, aperture_mrad=22.0,
                   defocus_ang=-20.0, kind=kind, potential_key=f"p{n}", calib_ang=0.25, targets=targets)


def _alone(srv, req):
    slices = srv.potentials[req.potential_key][:, :, :req.num_slices]
    modes = srv.probe(req.n, req.voltage_kv, req.aperture_mrad, req.calib_ang, req.defocus_ang, req.c3_ang)
    pos = torch.as_tensor(req.positions, device=srv.device)
    return pb.run_forward(slices, req.slice_thickness, modes, srv.weights, pos, req.voltage_kv, req.calib_ang,
                          req.calib_ang)


def test_single_job_equals_direct_forward(server):
    req = _req(128, 7, 19, seed=1)
    jid = server.submit(req)
    server.drain()
    res = server.finished[-1]
    assert res.state == _lib.JOB_DONE
    assert torch.equal(res.patterns, _alone(server, req))


def test_mixed_jobs_equal_alone(server):
    reqs = [_req(64, 5, 33, seed=2), _req(128, 12, 70, seed=3), _req(256, 3, 9, seed=4), _req(64, 20, 1, seed=5),
            _req(128, 1, 40, seed=6), _req(256, 9, 65, seed=7), _req(512, 5, 3, seed=10)]
    n0 = len(server.finished)
    # staggered: half submitted, a few ticks, then the rest join the running ones
    for r in reqs[:3]:
        server.submit(r)
    for _ in range(3):
        server.poll()
    for r in reqs[3:]:
        server.submit(r)
    server.drain()
    done = server.finished[n0:]
    assert len(done) == len(reqs)
    for res in done:
        assert res.state == _lib.JOB_DONE
        assert torch.equal(res.patterns, _alone(server, res.request))


def test_gradient_jobs_match_vjp_and_loss(server):
    n, s, p = 64, 6, 11
    req = _req(n, s, p, kind="grad", seed=8)
    clean = _alone(server, _req(n, s, p, seed=9))
    req.targets = clean * 1.1
    other = _req(128, 4, 17, seed=10)  # a forward job running alongside
    server.submit(other)
    server.submit(req)
    server.drain()
    res = [r for r in server.finished if r.request is req][0]
    assert res.state == _lib.JOB_DONE
    slices = server.potentials[req.potential_key][:, :, :s]
    modes = server.probe(n, req.voltage_kv, req.aperture_mrad, req.calib_ang, req.defocus_ang, req.c3_ang)
    pos = torch.as_tensor(req.positions, device=server.device)
    pat = _alone(server, req)
    assert torch.equal(res.patterns, pat)
    o = pat.detach().clone().requires_grad_(True)
    loss = amplitude_loss(o, req.targets)
    loss.backward()
    _, dv, dm = pb.vjp(slices, modes, server.weights, pos, o.grad, req.slice_thickness, req.voltage_kv,
                       req.calib_ang)
    rel = lambda a, b: float((a - b).norm() / b.norm())  # noqa: E731
    lv = loss.item()
    assert abs(res.loss.item() - lv) <= 1e-4 * lv
    assert rel(res.grad_potential, dv) < 1e-4
    assert rel(res.grad_modes, dm) < 1e-4


def test_rejects_malformed_and_oversized(server):
    with pytest.raises(ValueError):
        server.submit(_req(64, 5, 3, kind="grad"))  # gradient request without targets
    d = _lib.JobDesc()
    d.p = pb.simulations.ms_params(100, 5, 1, 3, 200.0, 1.95, 0.25, 0.25)  # unsupported grid edge
    with pytest.raises(ValueError):
        server.sched.submit(d)
    t = server.potentials["p256"]
    d3 = _lib.JobDesc()  # more probes in flight than the 512-slot budget
    d3.p = pb.simulations.ms_params(256, 24, 1, 4096, 200.0, 1.95, 0.25, 0.25, t.stride(), (256, 1, 1),
                                    batch=1024)
    d3.kind = _lib.PTYRO_JOB_FORWARD
    d3.potential = d3.modes = d3.weights = d3.positions = d3.patterns = t.data_ptr()
    with pytest.raises(ValueError, match="slot budget"):
        server.sched.submit(d3)


def test_cancel_queued_and_admission_waits_for_memory():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # an arena that holds one 256^2 job at a time: the others queue until it leaves
    srv = Server(arena_bytes=30 << 20, max_slots=256)
    rng = np.random.default_rng(1)
    srv.add_potential("p256", rng.uniform(0.0, 40.0, (256, 256, 8)).astype(np.float32))
    reqs = [Request(n=256, num_slices=8, positions=rng.uniform(-2, 2, (24, 2)), voltage_kv=200.0,
                    aperture_mrad=20.0, potential_key="p256", calib_ang=0.25, batch=16) for _ in range(3)]
    ids = [srv.submit(r) for r in reqs]
    # a job larger than the whole arena is rejected at submission (nothing is launched)
    big = _lib.JobDesc()
    pot = srv.potentials["p256"]
    big.p = pb.simulations.ms_params(256, 8, 1, 400, 200.0, 1.95, 0.25, 0.25, pot.stride(), (256, 1, 1), batch=200)
    big.kind = _lib.PTYRO_JOB_FORWARD
    big.potential = big.modes = big.weights = big.positions = big.patterns = pot.data_ptr()
    with pytest.raises(_lib.PtyroError, match="arena"):
        srv.sched.submit(big)
    srv.sched.step()
    states = [srv.sched.state(j) for j in ids]
    assert states[0] == _lib.JOB_RUNNING and _lib.JOB_QUEUED in states[1:]
    srv.sched.cancel(ids[2])
    assert srv.sched.state(ids[2]) == _lib.JOB_CANCELLED
    srv.drain()
    by_id = {id(r.request): r for r in srv.finished}
    assert by_id[id(reqs[0])].state == _lib.JOB_DONE and by_id[id(reqs[1])].state == _lib.JOB_DONE
    assert by_id[id(reqs[2])].state == _lib.JOB_CANCELLED
    free, slots = srv.sched.memory()
    assert slots == 256
    for r in reqs[:2]:
        want = _alone(srv, r)
        assert torch.equal(by_id[id(r)].patterns, want)
    srv.close()


def test_batch_plan_launch_and_graph_replay_equal_the_scheduler(server):
    """Uneven jobs (four grid edges, 2-6 slices, 1-7 probes, forward and gradient) as
    one recorded plan: a plain launch and a CUDA-graph replay give the scheduler's
    results bit for bit, and a replay reads the current contents of the inputs."""
    rng = np.random.default_rng(21)
    reqs = [_req(64, 5, 7, seed=31), _req(128, 3, 2, seed=32), _req(256, 2, 2, seed=33), _req(512, 2, 1, seed=35)]
    for n, s, p, seed in ((64, 4, 3, 34), (128, 6, 5, 36)):
        tg = torch.as_tensor(rng.uniform(0, 1e-3, (p, n, n)), dtype=torch.float32, device=server.device)
        reqs.append(_req(n, s, p, kind="grad", seed=seed, targets=tg))
    n0 = len(server.finished)
    for r in reqs:
        server.submit(r)
    server.drain()
    want = {id(res.request): res for res in server.finished[n0:]}
    assert all(res.state == _lib.JOB_DONE for res in want.values())

    def same(results):
        for r, res in zip(reqs, results):
            w = want[id(r)]
            assert torch.equal(res.patterns, w.patterns)
            if r.kind == "grad":
                assert torch.equal(res.grad_potential, w.grad_potential)
                assert torch.equal(res.grad_modes, w.grad_modes)
                assert torch.equal(res.loss, w.loss)

    plan, results = server.plan(reqs)
    plan.launch()
    torch.cuda.synchronize()
    plan.check()
    same(results)
    plan.capture()
    for res in results:
        res.patterns.zero_()
        if res.grad_potential is not None:
            res.grad_modes.zero_()
            res.loss.zero_()
    plan.replay()
    torch.cuda.synchronize()
    plan.check()
    same(results)
    # a replay recomputes from the inputs' current contents: move the first job's scan
    pos = plan._keep[0][2]
    pos.add_(0.75)
    plan.replay()
    torch.cuda.synchronize()
    r0 = reqs[0]
    moved = Request(n=r0.n, num_slices=r0.num_slices, positions=pos.cpu().numpy(), voltage_kv=r0.voltage_kv,
                    aperture_mrad=r0.aperture_mrad, defocus_ang=r0.defocus_ang, potential_key=r0.potential_key,
                    calib_ang=r0.calib_ang)
    assert torch.equal(results[0].patterns, _alone(server, moved))
    plan.close()
