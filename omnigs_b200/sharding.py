"""Data-parallel view sharding across GPUs (one process per GPU, torch.distributed).

The rasterizer's work splits naturally over views: every rank renders and back-propagates its own
views over a replicated Gaussian set, and one exchange follows per step -- the per-Gaussian
parameter gradients and the densification sums are added across ranks and the maximum radii are
max-reduced, after which every rank applies the same Adam step.  (The reference trains one view at
a time on one GPU, src/gaussian_mapper.cpp:290-440; its densification statistics are
gaussian_mapper.cpp:423-428.)

``assign_views`` balances views over ranks by pixel count (longest-processing-time first, ties by
view index, so every rank computes the same assignment); ``GradientReducer`` packs every summed
tensor into one flat buffer so a step costs one SUM all-reduce plus one MAX all-reduce of the radii
(NCCL over NVLink on GPUs, gloo on CPU).  Both collectives run on the caller's stream and can be
captured in the same CUDA graph as the step.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from .batch import BatchGradients


def assign_views(sizes, world: int) -> list[list[int]]:
    """Views (indices into ``sizes``, a list of (W, H)) for each of ``world`` ranks, balancing the
    pixel totals: views in decreasing pixel count each go to the least-loaded rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda v: (-sizes[v][0] * sizes[v][1], v))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for v in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(v)
        load[r] += sizes[v][0] * sizes[v][1]
    return [sorted(x) for x in out]


_SUM_FIELDS = ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations", "dL_dcolors", "dL_dcov3D",
               "grad_accum", "denom")


class GradientReducer:
    """Adds a rank's BatchGradients to every other rank's.  The summed tensors are views into one
    flat buffer (``flat``), so the exchange is a single all-reduce; ``max_radii`` is max-reduced.

    Densification sums accumulate across steps, so only this step's contribution may be added:
    ``reduce`` all-reduces the difference from the last reduced state, which it keeps.
    """

    def __init__(self, P: int, M: int, device, stats: bool = True, group=None):
        self.group = group
        shapes = {"dL_dmeans3D": (P, 3), "dL_dsh": (P, M, 3) if M else None, "dL_dopacity": (P, 1),
                  "dL_dscales": (P, 3), "dL_drotations": (P, 4), "dL_dcolors": None, "dL_dcov3D": None,
                  "grad_accum": (P, 1) if stats else None, "denom": (P, 1) if stats else None}
        sizes = {k: (0 if s is None else int(torch.Size(s).numel())) for k, s in shapes.items()}
        self.flat = torch.zeros(sum(sizes.values()), dtype=torch.float32, device=device)
        views, off = {}, 0
        for k in _SUM_FIELDS:
            n = sizes[k]
            views[k] = self.flat[off:off + n].view(shapes[k]) if n else None
            off += n
        self.grads = BatchGradients(max_radii=torch.zeros(P, device=device) if stats else None, **views)
        # running totals of the statistics as of the last reduce (after it)
        self._stats_prev = torch.zeros(2 * P if stats else 0, device=device)
        self.stats = stats
        self.P = P

    def _stat_span(self):
        k0 = self.grads.grad_accum
        base = self.flat.data_ptr()
        start = (k0.data_ptr() - base) // 4
        return start, start + 2 * self.P

    def reduce(self):
        """All-reduce this step's gradients (SUM) and the radii (MAX) across the group."""
        if self.stats:
            a, b = self._stat_span()
            # replace the accumulated statistics by this rank's contribution since the last reduce
            span = self.flat[a:b]
            span.sub_(self._stats_prev)
        dist.all_reduce(self.flat, op=dist.ReduceOp.SUM, group=self.group)
        if self.stats:
            span.add_(self._stats_prev)
            self._stats_prev.copy_(span)
            dist.all_reduce(self.grads.max_radii, op=dist.ReduceOp.MAX, group=self.group)
