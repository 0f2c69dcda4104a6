"""Multi-GPU bookkeeping for independent proofs (replicas; no data-path collective).

SALSAA proofs are independent, so N GPUs run N independent provers.  The only
cross-rank steps are a barrier around the timed region and the maximum of the
per-rank device times (the job is as slow as its slowest rank).  Seeds are
partitioned so that no two ranks prove the same statement.
"""
import os

SEED_STRIDE = 1 << 40


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment (1 GPU if absent)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def proof_seed(rank, step, slot, slots, base=1):
    """Seed of proof `slot` of batch `step` on `rank`: disjoint across ranks, steps and slots."""
    if not (0 <= slot < slots) or step < -(1 << 20) or step >= (1 << 30):
        raise ValueError("slot or step out of range")
    return base + rank * SEED_STRIDE + (step + (1 << 20)) * slots + slot


def max_over_ranks(value, device=None):
    """Max of a float over all ranks of the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
