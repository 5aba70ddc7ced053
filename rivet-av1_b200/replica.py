"""Replica plumbing: the post-filter chain on several GPUs of one node.

Frames and streams are independent units of the chain (the reference filters
one frame at a time, src/decoder/mod.rs:747-759, with no state carried from
frame to frame inside the filters), so N GPUs run N independent replicas: one
process per GPU, each filtering its own frames, with no collective on the
data path. The process group carries only control traffic: the barrier that
brackets a timed region and the max-over-ranks reduction of its elapsed time.

  Ranks                 rank/world/local from the torchrun environment, the
                        process group (nccl on GPUs, gloo on CPU), barrier()
                        and max() over ranks.
  shard                 the units a rank owns (round robin).
  assign_by_free_memory places streams on GPUs by free HBM, the admission
                        rule of the serving loop applied across devices.
  frame_seed            disjoint per-rank synthetic-input seeds.
"""
import datetime
import os

__all__ = ["Ranks", "shard", "assign_by_free_memory", "frame_seed", "aggregate_rate"]


class Ranks:
    """One process per GPU. `backend` None picks nccl when CUDA is usable,
    else gloo. With WORLD_SIZE 1 no process group is created and every
    operation is local."""

    def __init__(self, backend=None, timeout_s=300.0, env=None):
        env = os.environ if env is None else env
        self.rank = int(env.get("RANK", "0"))
        self.world = int(env.get("WORLD_SIZE", "1"))
        self.local = int(env.get("LOCAL_RANK", str(self.rank)))
        self.dist = None
        self.cuda = False
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.cuda = backend == "nccl"
            if self.cuda:
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            if dist.get_world_size() != self.world or dist.get_rank() != self.rank:
                raise RuntimeError("process group does not match RANK/WORLD_SIZE")
            self.dist = dist
        else:
            try:
                import torch
                self.cuda = torch.cuda.is_available()
            except ImportError:
                self.cuda = False

    def barrier(self):
        """All ranks reach this point; on GPUs the device is drained too, so a
        barrier on both sides of a timed region brackets finished work."""
        if self.cuda:
            import torch
            torch.cuda.synchronize()
        if self.dist:
            self.dist.barrier()
        if self.cuda:
            import torch
            torch.cuda.synchronize()

    def max(self, v):
        """The maximum of `v` over ranks (every rank gets it)."""
        if not self.dist:
            return float(v)
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        """The sum of `v` over ranks."""
        if not self.dist:
            return float(v)
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def shard(n_units, rank, world):
    """Indices of the units rank `rank` of `world` owns: round robin, so
    ranks' shares differ by at most one unit and mixed shapes spread evenly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(range(rank, n_units, world))


def assign_by_free_memory(demands, free):
    """Place streams on GPUs: stream i needs demands[i] bytes of HBM, GPU g
    has free[g] bytes. Streams are placed largest first, each on the GPU with
    the most free memory left (lowest index on ties), so the placement is
    deterministic. Returns the GPU index per stream; raises ValueError when a
    stream fits nowhere (the serving loop's admission refusal)."""
    left = list(free)
    out = [None] * len(demands)
    order = sorted(range(len(demands)), key=lambda i: (-demands[i], i))
    for i in order:
        g = max(range(len(left)), key=lambda k: (left[k], -k))
        if demands[i] > left[g]:
            raise ValueError(f"stream {i} needs {demands[i]} bytes; largest free is {left[g]}")
        left[g] -= demands[i]
        out[i] = g
    return out


def frame_seed(rank, i, base=1000):
    """Seed of the i-th synthetic frame of `rank` (distinct for i < base)."""
    if not 0 <= i < base:
        raise ValueError("frame index out of range")
    return base * (rank + 1) + i


def aggregate_rate(total_units, ms_max):
    """Whole-job rate: the units all ranks processed together / the slowest
    rank's time (ms), in units per second."""
    if ms_max <= 0:
        raise ValueError("elapsed time must be positive")
    return total_units / (ms_max / 1e3)
