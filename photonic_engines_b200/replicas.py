"""Several GPUs: one process per GPU (launched by torchrun), each an independent replica of the sampler.

Shots are independent chains, so the path shards with no exchange on the data path: every rank samples its
own shots with its own generator, and nothing crosses NVLink while sampling.  A collective appears only
where the caller asks for one: the MAX of device-timed figures, or every rank's occupations gathered onto
every rank.

    init(backend)                       process group from the torchrun environment, short timeout
    shard(total, world, rank)           the contiguous shot range [lo, hi) of a rank (strong scaling)
    replica_seed(seed, rank)            the generator seed of a rank's replica (disjoint Philox keys)
    max_over_ranks(x)                   a host float reduced with MAX over the ranks
    gather_rows(t)                      the ranks' [n_r, ...] tensors concatenated in rank order, on every rank
    sample_replicas(U, in_modes, total_shots, seed, ...)
                                        this rank's shard of a `total_shots` run (gathered on request)
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def world() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", device=None, timeout_s: float = 120.0) -> bool:
    """Join the process group of a torchrun launch (no-op for one process).  The timeout bounds every
    collective, so ranks waiting on a rank that died end with an error instead of hanging."""
    ws, _, _ = world()
    if ws <= 1 or dist.is_initialized():
        return dist.is_initialized()
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl" and device is not None:
        kw["device_id"] = torch.device(device)
    dist.init_process_group(backend, **kw)
    return True


def shard(total: int, world_size: int, rank: int) -> tuple[int, int]:
    """[lo, hi): rank r takes total // W shots, the first total % W ranks one more."""
    if world_size < 1 or not 0 <= rank < world_size or total < 0:
        raise ValueError(f"shard: total {total}, world {world_size}, rank {rank}")
    base, extra = divmod(total, world_size)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def replica_seed(seed: int, rank: int) -> int:
    """Seed of a rank's generator: distinct per rank, reproducible per (seed, rank)."""
    return (int(seed) * 1_000_003 + 7919 * int(rank) + 1) % (2 ** 63 - 1)


def _ready() -> bool:
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def _device_of_group():
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """MAX of a host float over the ranks (the time of a multi-GPU step is its slowest rank's)."""
    if not _ready():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_of_group())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(t: torch.Tensor) -> torch.Tensor:
    """Every rank's t [n_r, ...] concatenated in rank order (shards of different lengths allowed)."""
    if not _ready():
        return t
    dev = _device_of_group()
    n = torch.tensor([t.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(dist.get_world_size())]
    dist.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    top = max(sizes)
    pad = torch.zeros((top,) + tuple(t.shape[1:]), dtype=t.dtype, device=dev)
    pad[:t.shape[0]] = t.to(dev)
    parts = [torch.empty_like(pad) for _ in sizes]
    dist.all_gather(parts, pad)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)]).to(t.device)


def sample_replicas(U, in_modes, total_shots: int, seed: int, gather: bool = False, sampler=None, **kw):
    """This rank's shard of `total_shots` shots of U (rows lo..hi of the whole run), sampled with its own
    generator (`replica_seed`); gather=True returns all shards, in rank order, on every rank.  sampler
    defaults to `clifford.fock_sample`; extra keywords go to it."""
    if sampler is None:
        from .clifford import fock_sample as sampler
    ws, rank = (dist.get_world_size(), dist.get_rank()) if _ready() else (1, 0)
    lo, hi = shard(total_shots, ws, rank)
    dev = U.device if isinstance(U, torch.Tensor) else torch.device("cpu")
    gen = torch.Generator(device=dev).manual_seed(replica_seed(seed, rank))
    occ = sampler(U, in_modes, hi - lo, generator=gen, **kw)
    return gather_rows(occ) if gather else occ
