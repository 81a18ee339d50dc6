"""Sample sharding of one frame across ranks (one process per GPU).

Pixels and samples are independent units of the estimator: every rank renders its own samples
of the full frame with a seed offset that no other rank uses, and the per-rank sums are combined
with one all-reduce (NCCL over NVLink on GPUs, gloo on CPU).  Guiding state stays per rank, so
the combined estimator remains unbiased.
"""
import torch
import torch.distributed as dist

SEED_STRIDE = 1_000_003  # > any per-rank sample count between seed offsets; prime


def rank_seed(base_seed, rank, step):
    """Seed offset of `step` on `rank`: disjoint across ranks for steps < SEED_STRIDE."""
    if step >= SEED_STRIDE:
        raise ValueError("step exceeds the per-rank seed range")
    return (base_seed + rank * SEED_STRIDE + step) & 0xFFFFFFFF


def combine(sum_image, frames_per_rank, group=None):
    """All-reduces the per-rank sums of `frames_per_rank` frames and returns the mean image."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    out = sum_image.clone()
    if world > 1:
        dist.all_reduce(out, group=group)
    return out / float(frames_per_rank * world)


def render_sharded(render_frame, frames, base_seed=0, group=None, first_step=0):
    """render_frame(seed) -> image tensor; renders `frames` frames on this rank (steps first_step ..
    first_step + frames - 1 of its seed range) and returns the mean over all ranks' frames.  The
    per-rank sum is accumulated in place, and the ranks exchange it once, at the end."""
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    acc = None
    for k in range(frames):
        img = render_frame(rank_seed(base_seed, rank, first_step + k))
        if acc is None:
            acc = img.clone()
        else:
            acc.add_(img)
    return combine(acc, frames, group)
