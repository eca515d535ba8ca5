"""Replicas on the GPUs of one node: one process per GPU (launched by
torch.distributed.run), each encoding its own independent streams.

Frames of one stream depend on the previous frame's reconstruction, so a
stream never spans GPUs; streams, GOPs and frames of different streams share
nothing. The process group therefore carries no data: it lines the ranks up
(barrier) and takes the device time of the slowest rank (all-reduce MAX), and
whole-job throughput is the units every rank processed over that time.
"""
import os


def dist_env():
    """(world_size, rank, local_rank) from the launcher's environment; one
    process without it."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def stream_seeds(rank, streams):
    """Seeds of the synthetic streams that `rank` encodes: disjoint across
    ranks (at most 1000 streams per rank), so every rank's work is its own."""
    if not 0 <= streams <= 1000 or rank < 0:
        raise ValueError(f"rank {rank}, {streams} streams")
    return [rank * 1000 + s for s in range(streams)]


def aggregate_rate(world_size, units_per_rank, max_ms):
    """Whole-job throughput: the units all ranks processed (each the same
    number) over the slowest rank's time in milliseconds."""
    if max_ms <= 0:
        raise ValueError("time must be positive")
    return world_size * units_per_rank / (max_ms / 1000.0)


class Group:
    """The ranks' process group, or none for one process.

    backend "nccl" (one GPU per rank, device_id bound to LOCAL_RANK) or
    "gloo" (CPU); `device` is where the reduction tensor lives ("cuda" for
    nccl, "cpu" for gloo). Every rank must make the same calls in the same
    order; a short timeout makes ranks that wait for a missing peer fail
    instead of hanging."""

    def __init__(self, backend, device="cpu", timeout_s=120):
        self.world_size, self.rank, self.local = dist_env()
        self.device = device
        self.dist = None
        if self.world_size > 1:
            import datetime
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                import torch
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self, sync=None):
        """All ranks here; then `sync()` (the local device drained) if given."""
        if self.dist:
            self.dist.barrier()
        if sync:
            sync()

    def max(self, value):
        """The largest `value` over the ranks (every rank gets it)."""
        if not self.dist:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
