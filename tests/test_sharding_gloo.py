"""Multi-GPU protocol on CPU ranks (gloo, world size 2 and 3).

Each rank solves its contiguous path range with the global normalisation and
one all_reduce sums the partial results; the sum must equal one solve over
all paths.  The compute here is the FP64 oracle (the checker) injected as the
solver, so what is tested is the host protocol: the range split, the
normalisation and the reduction.  A rank that fails before the sum makes the
others fail within the process-group timeout instead of hanging.
"""
import os
import socket
import traceback

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cases import small_cases
from mcspeckle_b200 import mc as MC
from mcspeckle_b200.sharding import shard, sharded_cov, sharded_field

SEED = 2024


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_ranges_cover_exactly():
    for total in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            got = [shard(total, r, world, base_offset=5) for r in range(world)]
            assert sum(n for n, _ in got) == total
            off = 5
            for n, o in got:
                assert o == off
                off += n
            assert max(n for n, _ in got) - min(n for n, _ in got) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _oracle_field(h):
    from oracle import oracle
    return torch.from_numpy(oracle.field(h, oracle.Rng.philox()).reshape(-1, order="F").view(np.float64).copy())


def _oracle_cov(h):
    from oracle import oracle
    Ms, Mm = oracle.cov(h, oracle.Rng.philox())
    f = lambda x: torch.from_numpy(x.reshape(-1, order="F").view(np.float64).copy())  # noqa: E731
    return f(Ms), f(Mm)


def _worker(rank, world, port, case_idx, total, mode, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
        name, args, extra = small_cases(total)[case_idx]
        full_args = list(args) + list(extra)
        if mode == "fail" and rank == world - 1:
            raise RuntimeError("injected failure on the last rank before the reduction")
        u = sharded_field(full_args, total, seed=SEED, precision="fp64", solve=_oracle_field)
        Ms, Mm = sharded_cov(full_args, total, seed=SEED, precision="fp64", solve=_oracle_cov)
        if rank == 0:
            q.put(("ok", rank, u, Ms, Mm))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which decides
        q.put(("err", rank, f"{type(e).__name__}: {e}", traceback.format_exc()[-400:], None))


def _run(world, case_idx, total, mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, case_idx, total, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    alive = [p for p in ps if p.is_alive()]
    for p in alive:
        p.kill()
    out = []
    while not q.empty():
        out.append(q.get())
    return out, alive


@pytest.mark.parametrize("world,case_idx", [(2, 0), (3, 2), (2, 6)])
def test_sharded_sum_equals_one_solve(world, case_idx, oracle_lib):
    total = 301
    out, alive = _run(world, case_idx, total, "ok")
    assert not alive
    ok = [o for o in out if o[0] == "ok"]
    assert ok, out
    _, _, u, Ms, Mm = ok[0]
    name, args, extra = small_cases(total)[case_idx]
    h = MC.mc_args(*(list(args) + list(extra)), seed=SEED, precision="fp64")
    u1 = oracle_lib.field(h, oracle_lib.Rng.philox())
    Ms1, Mm1 = oracle_lib.cov(h, oracle_lib.Rng.philox())
    rel = lambda a, b: np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())  # noqa: E731
    assert rel(u, u1) < 1e-12
    assert rel(Ms, Ms1) < 1e-12 and rel(Mm, Mm1) < 1e-12


def test_failed_rank_does_not_hang_the_others():
    out, alive = _run(2, 0, 101, "fail")
    assert not alive, "a rank hung waiting for a failed peer"
    errs = {o[1]: o[2] for o in out if o[0] == "err"}
    assert 1 in errs and "injected failure" in errs[1]
    assert 0 in errs  # the surviving rank's collective ended with an error
