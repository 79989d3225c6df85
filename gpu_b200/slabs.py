"""The reference's multi-GPU SART with one z-slab per process.

The reference's default build (V63/main_recon.cu:23, Number_of_Devices 4)
drives its devices from one host thread
(V63/host_IterativeRecon_CBCT_multiGPU.c:1-161): per view every device
projects its slab into partial ray sums, the host adds the parts in device
order and divides, and every device backprojects the one correction into its
slab.  Here the devices are ``torch.distributed`` ranks, one GPU each: rank r
holds slab r, the parts are exchanged by an all-gather (NCCL over NVLink on
GPUs), and every rank combines all parts itself, in rank order, so every
rank holds the same correction -- the reference's -- without a broadcast.
Per view and rank the exchange is rows*nu*2 floats (6 MiB at 1024x768).

The per-view steps are the C ABI's ``ctr_forward_partial``,
``ctr_combine_partials`` and ``ctr_sart_update``; ``SlabOps`` binds them to a
slab geometry.  The driver takes any object with the same three methods, so
its exchange and ordering logic also runs on CPU tensors.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from .ctrecon import Geometry, GeometryDesc, VOLUME_TILED


class SlabOps:
    """The per-view steps of one slab on the current GPU."""

    def __init__(self, desc: GeometryDesc, n_slabs: int, slab: int):
        self.geom = Geometry(desc, n_slabs, slab)

    @property
    def vol_shape(self):
        return self.geom.vol_shape

    @property
    def view_shape(self):
        return self.geom.view_shape

    def forward_partial(self, vol, view, part, tiled=False):
        self.geom.forward_partial(vol, view, part, VOLUME_TILED if tiled else 0)

    def combine(self, parts, view, b_view, rays):
        self.geom.combine_partials(parts, view, b_view, rays)

    def update(self, vol, rays, view, beta, flags=0, seed=0, tiled=False):
        self.geom.sart_update(vol, rays, view, beta, flags | (VOLUME_TILED if tiled else 0), seed)


def exchange(part: torch.Tensor, parts: torch.Tensor, group=None):
    """parts[r] <- rank r's part, for every rank r of the group."""
    if dist.get_backend(group) == "nccl":
        dist.all_gather_into_tensor(parts, part, group=group)
    else:
        dist.all_gather(list(parts.unbind(0)), part, group=group)


class SlabSART:
    """SART views of one rank's slab (rank r of world_size holds slab r)."""

    def __init__(self, ops, rank: int, world_size: int, device, group=None):
        self.ops, self.rank, self.world, self.group = ops, rank, world_size, group
        rows, nu = ops.view_shape
        self.part = torch.zeros((rows, nu, 2), dtype=torch.float32, device=device)
        self.parts = torch.zeros((world_size, rows, nu, 2), dtype=torch.float32, device=device)
        self.rays = torch.zeros((rows, nu, 2), dtype=torch.float32, device=device)

    def views(self, vol, sino, beta, view_begin, view_count, flags=0, seed=0, tiled=False):
        """vol: this rank's slab; sino: the whole sinogram (every rank combines every ray)."""
        for j in range(view_begin, view_begin + view_count):
            self.ops.forward_partial(vol, j, self.part, tiled=tiled)    # multiGPU.c:71-75
            exchange(self.part, self.parts, self.group)                # :86-91, the parts of all devices
            self.ops.combine(self.parts, j, sino[j], self.rays)        # :82-95, in device order
            self.ops.update(vol, self.rays, j, beta, flags, seed, tiled=tiled)   # :103-112
        return vol


def slab_of(vol: torch.Tensor, rank: int, world_size: int) -> torch.Tensor:
    """Rank's slab of a whole [z][y][x] volume (a view, no copy)."""
    zs = vol.shape[0] // world_size
    return vol[zs * rank: zs * (rank + 1)]


__all__ = ["SlabOps", "SlabSART", "exchange", "slab_of"]
