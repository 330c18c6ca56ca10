"""Losses and value-and-gradient helpers for ptychographic reconstruction.

The reference's reconstruction loops (``src/ptyrodactyl/multislice/multislice_recon.py``)
reduce simulated against measured intensities with ``_reduce_loss`` (MAE, MSE or RMSE,
``:127-163``) and take ``jax.value_and_grad`` through ``stem_4d`` (``:1940``). The
same reductions are provided here, plus the amplitude loss of Gauss-Newton /
Levenberg-Marquardt ptychography, and :func:`value_and_grad` returns the loss with
its gradients w.r.t. the potential and the probe aberrations, the derivative
flowing through the engine's adjoint kernel.
"""

from __future__ import annotations

from typing import Dict, Optional

import torch

from .autodiff import make_probe_differentiable, stem_4d_patterns


def reduce_loss(model: torch.Tensor, data: torch.Tensor, mode: str = "mse") -> torch.Tensor:
    """_reduce_loss (multislice_recon.py:127-163): mean absolute, mean squared or root
    mean squared error of intensities."""
    diff = model - data
    if mode == "mae":
        return diff.abs().mean()
    if mode == "mse":
        return (diff * diff).mean()
    if mode == "rmse":
        return torch.sqrt((diff * diff).mean())
    raise ValueError(f"unknown loss mode: {mode}")


def amplitude_loss(model: torch.Tensor, data: torch.Tensor, eps: float = 1e-12) -> torch.Tensor:
    """sum (sqrt(I_model) - sqrt(I_measured))^2 over all patterns and pixels."""
    return ((torch.sqrt(model + eps) - torch.sqrt(torch.clamp(data, min=0.0))) ** 2).sum()


def value_and_grad(field: torch.Tensor, aberrations: Dict[str, torch.Tensor], targets: torch.Tensor,
                   windows: Optional[torch.Tensor], positions: torch.Tensor, *, n: int, voltage_kv: float,
                   aperture_mrad: float, calib_ang: float, slice_thickness: float, c5_ang: float = 0.0,
                   loss: str = "amplitude", ckpt_every: int = 0, batch: int = 0):
    """Loss and its gradients for potential ``field`` (F, F, S) and the probe
    aberrations (keys ``defocus``, ``c3``, ``a1x``, ``a1y``; scalar tensors).

    Returns (loss, dL/dfield, {name: dL/dname}). Probe p reads the n x n window of the
    field at ``windows[p]`` (or the whole field if ``windows`` is None and F == n).
    """
    field = field.detach().requires_grad_(True)
    ab = {k: v.detach().to(torch.float64).requires_grad_(True) for k, v in aberrations.items()}
    probe = make_probe_differentiable(voltage_kv, aperture_mrad, (n, n), calib_ang * 100.0,
                                      ab.get("defocus", 0.0), ab.get("c3", 0.0), c5_ang, ab.get("a1x", 0.0),
                                      ab.get("a1y", 0.0), device=field.device)
    modes = probe[..., None].contiguous()
    weights = torch.ones(1, dtype=torch.float32, device=field.device)
    pat = stem_4d_patterns(field, modes, weights, positions, slice_thickness, voltage_kv, calib_ang,
                           ckpt_every=ckpt_every, batch=batch, windows=windows)
    value = amplitude_loss(pat, targets) if loss == "amplitude" else reduce_loss(pat, targets, loss)
    value.backward()
    grads = {k: v.grad.detach() for k, v in ab.items()}
    return value.detach(), field.grad.detach(), grads


def sharded_value_and_grad(field: torch.Tensor, aberrations: Dict[str, torch.Tensor], targets: torch.Tensor,
                           windows: Optional[torch.Tensor], positions: torch.Tensor, *, group=None,
                           local_fn=None, **kwargs):
    """value_and_grad over scan positions sharded across the ranks of a
    torch.distributed process group (one process per GPU, NCCL over NVLink): each
    rank passes its own probes (positions, targets, windows), runs the forward and
    the adjoint kernels on them, and one all-reduce per quantity sums the loss, the
    potential gradient and the aberration gradients — the only exchange of the
    sharded path (the reference shards positions the same way,
    multislice/parallelized.py:512-521). Mean-type losses are weighted by each
    rank's share of the patterns before the sum. ``local_fn`` replaces the local
    computation (tests)."""
    import torch.distributed as dist
    fn = value_and_grad if local_fn is None else local_fn
    value, g_field, g_ab = fn(field, aberrations, targets, windows, positions, **kwargs)
    if not dist.is_available() or not dist.is_initialized():
        return value, g_field, g_ab
    world = dist.get_world_size(group)
    loss = kwargs.get("loss", "amplitude")
    if loss in ("mae", "mse", "rmse") and world > 1:
        count = torch.tensor([float(targets.numel())], dtype=torch.float64, device=g_field.device)
        total = count.clone()
        dist.all_reduce(total, group=group)
        share = float(count.item() / total.item())
        if loss == "rmse":  # combine mean squares, then the root: d sqrt(m)/dm = 1 / (2 sqrt(m))
            ms = value.to(torch.float64) ** 2 * share
            g_scale = share * value.to(torch.float64)  # dL_r/dx = dms_r/dx / (2 L_r); rescaled below
            buf = ms.reshape(1).to(g_field.device)
            dist.all_reduce(buf, group=group)
            root = torch.sqrt(buf)[0]
            scale = (g_scale / root).to(g_field.dtype)
            value = root.to(value.dtype)
            g_field = g_field * scale
            g_ab = {k: v * scale.to(v.dtype) for k, v in g_ab.items()}
        else:
            value = value * share
            g_field = g_field * share
            g_ab = {k: v * share for k, v in g_ab.items()}
    if loss != "rmse" or world == 1:
        v = value.reshape(1).to(g_field.device).clone()
        dist.all_reduce(v, group=group)
        value = v[0]
    g_field = g_field.contiguous()
    dist.all_reduce(g_field, group=group)
    names = sorted(g_ab)
    if names:
        flat = torch.stack([g_ab[k].reshape(()).to(torch.float64) for k in names]).to(g_field.device)
        dist.all_reduce(flat, group=group)
        g_ab = {k: flat[i] for i, k in enumerate(names)}
    return value, g_field, g_ab
