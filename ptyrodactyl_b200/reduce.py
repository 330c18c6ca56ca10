"""The late distribution reducers of the detector path (multislice/reduce.py):
one ``|.|^2`` per reduction, coherent axes summed inside it and incoherent axes
outside it.

``bound_amplitude_fn`` maps one float64 sample row (a 1-D tensor) to one complex
(H, W) field, on any device. The reducers are plain torch: differentiable in the
distributions' weights and in whatever the bound function closes over. The engine's
own ensemble path (``ensemble.py``) performs the same reductions inside its kernels;
these are the public building blocks for callers who bind their own amplitude
kernels, as the reference's are.
"""

from __future__ import annotations

from typing import Callable, Sequence

import torch

from .types import Distribution, ReductionMode

BoundAmplitude = Callable[[torch.Tensor], torch.Tensor]


def _weighted_sum(field: torch.Tensor, weights: torch.Tensor, axis: int) -> torch.Tensor:
    w = weights.to(device=field.device, dtype=field.dtype)
    shape = [1] * field.ndim
    shape[axis] = w.shape[0]
    return (field * w.reshape(shape)).sum(dim=axis)


def apply_distribution(distribution: Distribution, bound_amplitude_fn: BoundAmplitude) -> torch.Tensor:
    """reduce.py:29-90: ``|sum_n w_n A(s_n)|^2`` for a COHERENT axis,
    ``sum_n w_n |A(s_n)|^2`` for an INCOHERENT one; (H, W) real."""
    amplitudes = torch.stack([bound_amplitude_fn(row) for row in distribution.samples])
    if distribution.reduction is ReductionMode.COHERENT:
        return _weighted_sum(amplitudes, distribution.weights, 0).abs() ** 2
    if distribution.reduction is ReductionMode.INCOHERENT:
        return _weighted_sum(amplitudes.abs() ** 2, distribution.weights, 0)
    raise ValueError("unknown distribution reduction mode")


def apply_distributions(distributions: Sequence[Distribution], bound_amplitude_fn: BoundAmplitude) -> torch.Tensor:
    """reduce.py:93-201: ``sum_i prod(w_i) |sum_c prod(w_c) A(concat rows)|^2`` over
    the Cartesian product of the axes' samples. The bound function receives the
    concatenation of one row of each axis, in tuple order; coherent axes are reduced
    inside the modulus (last axis first), incoherent axes outside it."""
    distributions = tuple(distributions)
    if len(distributions) == 0:
        raise ValueError("distributions must contain at least one axis")
    counts = tuple(int(d.samples.shape[0]) for d in distributions)
    grids = torch.meshgrid(*[torch.arange(c) for c in counts], indexing="ij")
    rows = torch.cat([d.samples[g.reshape(-1)] for d, g in zip(distributions, grids)], dim=1)
    flat = torch.stack([bound_amplitude_fn(row) for row in rows])
    field = flat.reshape(counts + tuple(flat.shape[1:]))
    labels = list(range(len(distributions)))
    for axis in sorted((i for i, d in enumerate(distributions) if d.reduction is ReductionMode.COHERENT),
                       reverse=True):
        cur = labels.index(axis)
        field = _weighted_sum(field, distributions[axis].weights, cur)
        labels.pop(cur)
    intensity = field.abs() ** 2
    for axis in sorted((i for i, d in enumerate(distributions) if d.reduction is ReductionMode.INCOHERENT),
                       reverse=True):
        cur = labels.index(axis)
        intensity = _weighted_sum(intensity, distributions[axis].weights, cur)
        labels.pop(cur)
    return intensity
