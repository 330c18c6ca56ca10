"""The sharded gradient's exchange on CPU: two gloo ranks, each with a stand-in
local gradient, must end with the global loss and gradients."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local(rank):
    def fn(field, aberrations, targets, windows, positions, **kw):
        # loss = sum over this rank's targets of (field.sum() * t)^2 / 2, a shard-additive stand-in
        f = field.detach().clone().requires_grad_(True)
        ab = {k: v.detach().clone().requires_grad_(True) for k, v in aberrations.items()}
        model = f.sum() * targets + ab["defocus"] * positions[:, 0]  # one value per probe
        if kw.get("loss") == "mse":
            val = (model ** 2).mean()
        elif kw.get("loss") == "rmse":
            val = torch.sqrt((model ** 2).mean())
        else:
            val = (model ** 2).sum() / 2
        val.backward()
        return val.detach(), f.grad, {k: v.grad for k, v in ab.items()}
    return fn


def _worker(rank, world, port, loss, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from ptyrodactyl_b200.recon import sharded_value_and_grad
        g = torch.Generator().manual_seed(3)
        field = torch.randn(4, 4, 2, generator=g, dtype=torch.float64)
        targets = torch.randn(6, generator=g, dtype=torch.float64)
        positions = torch.randn(6, 2, generator=g, dtype=torch.float64)
        shard = slice(rank * 3, rank * 3 + 3)
        ab = {"defocus": torch.tensor(0.3, dtype=torch.float64)}
        val, gf, gab = sharded_value_and_grad(field, ab, targets[shard], None, positions[shard],
                                              local_fn=_local(rank), loss=loss)
        # the same quantity computed on all probes at once
        ref_v, ref_g, ref_ab = _local(0)(field, ab, targets, None, positions, loss=loss)
        ok = (abs(float(val) - float(ref_v)) < 1e-10 and torch.allclose(gf, ref_g, atol=1e-10) and
              abs(float(gab["defocus"]) - float(ref_ab["defocus"])) < 1e-10)
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("loss", ["amplitude", "mse", "rmse"])
def test_sharded_gradient_sums_over_ranks(loss):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, loss, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    results = dict(q.get(timeout=10) for _ in procs)
    assert all(p.exitcode == 0 for p in procs)
    assert results == {0: True, 1: True}
