"""Replicas over GPUs: one process per GPU under torchrun (torch.distributed).

The path does not shard: every system of a batch is independent and a batch
fits one GPU.  N GPUs therefore run N independent replicate ensembles, each
with its own shifted Philox seeds, and the only collectives are a barrier
around the timed region and the max-over-ranks reduction of its duration.
These helpers hold that plumbing so that it runs the same way on NCCL (GPU)
and on gloo (the CPU tests).
"""
import datetime
import os

SEED_STRIDE = 7919      # seed shift between ranks (prime, so no two systems of two ranks coincide)


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, timeout_s=120):
    """Join the process group when there is more than one rank."""
    import torch.distributed as dist
    ws, _, _ = env()
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws > 1


def replica_boxes(boxes, rank):
    """The batch's boxes with this rank's seeds."""
    return [(lo, hi, per, sd + SEED_STRIDE * rank) for (lo, hi, per, sd) in boxes]


def replica_seed(seed, rank):
    """The seed of a single-system handle on this rank."""
    return seed + rank


def barrier(cuda_sync=True):
    import torch
    import torch.distributed as dist
    if cuda_sync and torch.cuda.is_available():
        torch.cuda.synchronize()
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(x, device="cpu"):
    """The maximum of a per-rank float over all ranks."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(n_per_rank, ranks, steps, seconds_max):
    """Whole-job particle-steps/s: all ranks' particle-steps over the slowest rank's time."""
    return n_per_rank * ranks * steps / seconds_max


def finalize():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
