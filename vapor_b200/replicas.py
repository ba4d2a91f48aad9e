"""Host logic of the replica mode (`bench.py --gpus N`): one independent scene
per rank, no collective on the data path; ranks meet only at barriers and in
the max-over-ranks reduction of their timings."""
import os


def rank_info():
    """(world, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def scene_seed(base, rank):
    """Seed of this rank's scene: every replica runs its own plume."""
    return int(base) + int(rank)


def max_over_ranks(value, dist=None, device=None):
    """The maximum of a per-rank scalar over all ranks (the job's time is the
    slowest rank's). Without a process group it is the value itself."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_steps_per_second(world, steps, max_ms):
    """Whole-job throughput: all ranks' steps over the slowest rank's time."""
    return world * steps / (max_ms * 1e-3)
