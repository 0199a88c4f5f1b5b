"""Multi-GPU sharding of one MCfield / MCcov solve: one process per GPU.

Paths are independent (each draws from its own Philox stream), so a solve of
P paths splits into contiguous path ranges, one per rank.  Every rank solves
its range with the normalisation of the whole solve (norm_itr = P), then one
sum over ranks (torch.distributed all_reduce: NCCL over NVLink for CUDA
tensors, gloo for host tensors) gives exactly the single-process result.
This is the parfor reduction of scmc.m:443-444 and 496-498 with
MCfield.m:253-254 / MCcov.m:293-299 applied once, globally.  No data moves
between GPUs other than that final sum.

The solver is pluggable: by default the CUDA library (device outputs, so the
sum runs on the GPU); tests substitute a host solver to check the range
split, the normalisation and the reduction on CPU ranks.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from . import mc as _mc


def shard(total: int, rank: int, world: int, base_offset: int = 0):
    """(paths, path_offset) of `rank`: contiguous ranges, the first
    total % world ranks one path longer."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    q, r = divmod(int(total), world)
    n = q + (1 if rank < r else 0)
    off = base_offset + rank * q + min(rank, r)
    return n, off


def _args_for(args, n, seed, precision, device, off, total):
    a = list(args)
    a[8] = n
    return _mc.mc_args(*a, seed=seed, precision=precision, device=device, path_offset=off, norm_itr=total)


def _gpu_field(h):
    import torch
    a = h.args
    u = torch.empty(2 * a.nv * a.nl, dtype=torch.float64, device=f"cuda:{a.device}")
    st = torch.cuda.current_stream(a.device)
    _lib.check(_lib.lib().scmc_field_device(h.ref, u.data_ptr(), st.cuda_stream))
    return u


def _gpu_cov(h):
    import torch
    a = h.args
    n = 2 * (a.nv * a.nl) ** 2
    Ms = torch.empty(n, dtype=torch.float64, device=f"cuda:{a.device}")
    Mm = torch.empty(n, dtype=torch.float64, device=f"cuda:{a.device}")
    st = torch.cuda.current_stream(a.device)
    _lib.check(_lib.lib().scmc_cov_device(h.ref, Ms.data_ptr(), Mm.data_ptr(), st.cuda_stream))
    return Ms, Mm


def sharded_field(args, total, *, seed, precision="mixed", device=0, group=None, solve=None):
    """MCfield positional args (maxItr ignored; `total` paths) split over the
    ranks of `group`.  Returns u (nv x nl complex, numpy) on every rank."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n, off = shard(total, rank, world)
    h = _args_for(args, n, seed, precision, device, off, total)
    u = (solve or _gpu_field)(h)
    dist.all_reduce(u, group=group)
    a = h.args
    return u.cpu().numpy().view(np.complex128).reshape(a.nv, a.nl, order="F")


def sharded_cov(args, total, *, seed, precision="mixed", device=0, group=None, solve=None):
    """MCcov split over the ranks of `group`; returns (Ms, Mm) on every rank."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n, off = shard(total, rank, world)
    h = _args_for(args, n, seed, precision, device, off, total)
    Ms, Mm = (solve or _gpu_cov)(h)
    dist.all_reduce(Ms, group=group)
    dist.all_reduce(Mm, group=group)
    a = h.args
    shp = (a.nv, a.nv, a.nl, a.nl)
    return tuple(x.cpu().numpy().view(np.complex128).reshape(shp, order="F") for x in (Ms, Mm))
