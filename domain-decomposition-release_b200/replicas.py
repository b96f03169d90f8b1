"""Shot replicas over several GPUs.

Shots are independent, so each process (one per GPU) holds the whole model
and migrates its own share of the shots into its own stacks; the only
exchange is one sum of the five FP64 stacks at the end of the job, before
the Laplacian and the source compensation (the reference applies both to
the stack of all shots, RTM/rtm3d_1_model_mpi_blend/
rtm3d_blend_elastic_model_mpi_meat.hpp:115-124, where
RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/
elastic_1_rtm3d_model_mpi).  The reference splits one model into
subdomains over MPI ranks instead; a B200 holds the whole model, so no
halo exchange exists here.

The sum runs through ``torch.distributed``: on CUDA tensors over NCCL when
the process group's backend is ``nccl`` (the stacks move device to device,
``jv_image_get_device`` / ``jv_image_set_device``), on host tensors
otherwise (``gloo``).  Every rank takes the same collective steps in the
same order.
"""
from __future__ import annotations

from typing import Callable, Iterable, Optional, Sequence

import numpy as np

N_KINDS = 5  # ip, pp, ps, sp, ss (IMG_IP .. IMG_SS)


def shard_shots(n_shot: int, rank: int, world: int) -> list:
    """Shots of `rank`: round robin (shot s runs on rank s % world), so
    every shot runs exactly once and ranks differ by at most one shot."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n_shot < 0:
        raise ValueError("n_shot must be >= 0")
    return list(range(rank, n_shot, world))


def migrate_shots(ctx, shots: Iterable[int],
                  observed: Optional[Callable[[int], Sequence[np.ndarray]]] = None) -> int:
    """Migrates `shots` into ctx's stacks.  `observed(shot)` returns the
    shot's (vx, vy, vz) traces; without it each shot is modelled first on
    the same context, as the reference's RTM job does
    (rtm3d_blend_elastic_model_mpi_meat.hpp:22-38, 50-113).  Returns the
    number of shots migrated."""
    n = 0
    for s in shots:
        obs = observed(s) if observed is not None else ctx.forward(s)
        ctx.rtm_shot(s, obs)
        n += 1
    return n


def reduce_images(ctx, group=None, device: Optional[int] = None) -> None:
    """Sums the five stacks of `ctx` over the ranks of `group` and loads
    the sum back into every rank's context, so that ``finalize`` on any
    rank gives the image of all shots."""
    import torch
    import torch.distributed as dist

    n = int(ctx.info().n_phy)
    on_gpu = dist.get_backend(group) == "nccl"
    if on_gpu:
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        buf = torch.empty((N_KINDS, n), dtype=torch.float64, device=dev)
        for k in range(N_KINDS):
            ctx.image_to_device(k, buf[k].data_ptr())  # returns after the copy has finished
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        torch.cuda.synchronize(dev)  # the library copies on its own stream
        for k in range(N_KINDS):
            ctx.image_from_device(k, buf[k].data_ptr())
    else:
        buf = torch.empty((N_KINDS, n), dtype=torch.float64)
        for k in range(N_KINDS):
            buf[k].copy_(torch.from_numpy(np.ascontiguousarray(ctx.image(k)).reshape(-1)))
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        for k in range(N_KINDS):
            ctx.set_image(k, buf[k].numpy())


def run_job(ctx, n_shot: int, group=None,
            observed: Optional[Callable[[int], Sequence[np.ndarray]]] = None) -> list:
    """The whole replica job on one rank: zero the stacks, migrate this
    rank's shots, sum the stacks over the group.  Returns this rank's
    shots."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = shard_shots(n_shot, rank, world)
    ctx.image_reset()
    migrate_shots(ctx, mine, observed)
    reduce_images(ctx, group)
    return mine
