"""The request server (scmc_server_*): continuous batching of MCfield /
MCcov solves on worker slots with their own streams and scratch.

Each request's result must be the same alone (scmc_field / scmc_cov on the
library's default context) and in the mix (on a server slot, overlapping
other requests): every path draws from its own Philox stream and every
accumulator is private, so only the order of sums may differ: of FP64 atomic
sums in FP64 mode (tolerance 1e-12 relative), and in the reduced precisions
also the order in which the one-pass walk writes its records, which decides
which events share an FP32 tensor-core chunk (tolerance 1e-6; 1e-4 for the
900 x 200 request of 20 000 paths, whose FP32 chunk sums run over tens of
thousands of events each, so their rounding depends on the order at about
1e-5 relative).  Also: admission never reserves more than the
HBM budget, oversize requests are refused, a failing request does not disturb
the others, and destroying the server cancels what is still queued.
"""
import numpy as np
import pytest

from mcspeckle_b200 import _abi, _lib
from mcspeckle_b200 import workloads as WL
from mcspeckle_b200 import mc as MC
from mcspeckle_b200.serving import Server

pytestmark = pytest.mark.gpu

SAME_TOL = 1e-12
SAME_TOL_MIXED = 1e-6
SAME_TOL_MIXED_LARGE = 1e-4


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def small_stream(n=24, seed=3):
    return WL.served_requests(n, seed=seed, paths=(200, 3000), nv_max=160, nl_max=64, side_mfp=(5.0, 12.0))


def holder(r, precision="mixed"):
    return MC.mc_args(*r["args"], seed=r["seed"], precision=precision)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_same_alone_and_in_the_mix(gpu, precision):
    reqs = small_stream()
    assert any(r["nv"] >= 64 and r["nl"] >= 32 for r in reqs)  # some take the tensor-core field path
    with Server(slots=6) as srv:
        tickets = [srv.submit_field(holder(r, precision)) for r in reqs]
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    slots = {info["slot"] for _, info in mixed}
    assert len(slots) > 1
    # requests overlapped in time on different slots
    iv = sorted((info["start_ms"], info["done_ms"]) for _, info in mixed)
    assert any(iv[k + 1][0] < iv[k][1] for k in range(len(iv) - 1))
    for r, (u, info) in zip(reqs, mixed):
        alone = MC.field_from_args(holder(r, precision))
        assert u.shape == alone.shape == (r["nv"], r["nl"])
        assert rel(u, alone) < (SAME_TOL if precision == "fp64" else SAME_TOL_MIXED)
        assert info["status"] == 0 and info["finished"] == 1
        assert info["done_ms"] >= info["start_ms"] >= info["submit_ms"]
        assert info["peak_bytes"] <= info["reserved_bytes"]


def test_cov_requests_in_the_mix(gpu):
    reqs = small_stream(6, seed=9)
    cov_args = WL.cov64_args(400)
    cov_args[4] = WL.grid_rect(4, 4, 5.0, +1.0)
    cov_args[5] = WL.grid_rect(4, 4, 5.0, -1.0)
    hc = MC.mc_args(*cov_args, seed=77, precision="mixed")
    with Server(slots=3) as srv:
        tf = [srv.submit_field(holder(r)) for r in reqs[:3]]
        tc = srv.submit_cov(hc)
        tf += [srv.submit_field(holder(r)) for r in reqs[3:]]
        (Ms, Mm), info = srv.wait(tc)
        fields = [srv.wait(t)[0] for t in tf]
    Ms0, Mm0 = MC.cov_from_args(hc)
    assert rel(Ms, Ms0) < SAME_TOL_MIXED and rel(Mm, Mm0) < SAME_TOL_MIXED
    for r, u in zip(reqs, fields):
        assert rel(u, MC.field_from_args(holder(r))) < SAME_TOL_MIXED


def test_budget_admission(gpu):
    """With a budget that fits only the largest request alone, requests whose
    reservations add up to more than the budget never run at the same time."""
    reqs = small_stream(8, seed=4)
    with Server(slots=4) as srv:
        first = [srv.wait(srv.submit_field(holder(r)))[1] for r in reqs]
    budget = 1.05 * max(i["reserved_bytes"] for i in first)
    with Server(slots=4, hbm_budget=budget) as srv:
        tickets = [srv.submit_field(holder(r)) for r in reqs]
        out = [srv.wait(t)[1] for t in tickets]
        st = srv.stats()
    assert st["peak_reserved_bytes"] <= st["budget_bytes"]
    pairs = 0
    for i in range(len(out)):
        for j in range(i + 1, len(out)):
            a, b = out[i], out[j]
            if a["reserved_bytes"] + b["reserved_bytes"] > st["budget_bytes"]:
                pairs += 1
                assert a["done_ms"] <= b["start_ms"] or b["done_ms"] <= a["start_ms"]
    assert pairs > 0


def test_oversize_request_refused(gpu):
    cov_args = WL.cov64_args(100)
    h = MC.mc_args(*cov_args, seed=1, precision="mixed")  # 64x64 cov: ~1 GB of accumulators
    with Server(slots=2, hbm_budget=2e8) as srv:
        with pytest.raises(_lib.ScmcError) as ei:
            srv.submit_cov(h)
        assert ei.value.status == _abi.SCMC_ERR_NOMEM


def test_failing_request_isolated(gpu):
    reqs = small_stream(5, seed=6)
    bad = MC.mc_args(*reqs[0]["args"], seed=1, precision="mixed", max_events_per_path=1)
    with Server(slots=2) as srv:
        t_ok1 = srv.submit_field(holder(reqs[1]))
        t_bad = srv.submit_field(bad)
        t_ok2 = srv.submit_field(holder(reqs[2]))
        with pytest.raises(_lib.ScmcError) as ei:
            srv.wait(t_bad)
        assert ei.value.status == _abi.SCMC_ERR_LIMIT
        u1, _ = srv.wait(t_ok1)
        u2, _ = srv.wait(t_ok2)
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 2
    assert rel(u1, MC.field_from_args(holder(reqs[1]))) < SAME_TOL_MIXED
    assert rel(u2, MC.field_from_args(holder(reqs[2]))) < SAME_TOL_MIXED


def test_poll_and_destroy_with_queue(gpu):
    reqs = small_stream(12, seed=8)
    srv = Server(slots=1)
    tickets = [srv.submit_field(holder(r)) for r in reqs]
    while not srv.poll(tickets[0]):
        pass
    u0, info0 = srv.wait(tickets[0])
    assert info0["finished"] == 1
    srv.close()  # runs the admitted request to completion, cancels the queue
    assert rel(u0, MC.field_from_args(holder(reqs[0]))) < SAME_TOL_MIXED


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_small_requests_are_packed(gpu, precision):
    """Small CUDA-core field requests submitted together run in packs (one walk,
    accumulation and finalisation per round for many requests), with the same
    results as each request alone."""
    reqs = WL.served_requests(40, seed=21, paths=(300, 5000), nv_max=48, nl_max=24, side_mfp=(5.0, 12.0))
    with Server(slots=2) as srv:
        tickets = [srv.submit_field(holder(r, precision)) for r in reqs]
        out = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    sizes = [info["packed"] for _, info in out]
    assert max(sizes) > 4  # many requests shared their launches
    for r, (u, info) in zip(reqs, out):
        alone = MC.field_from_args(holder(r, precision))
        assert rel(u, alone) < (SAME_TOL if precision == "fp64" else SAME_TOL_MIXED)


def test_large_head_does_not_block_small_requests(gpu):
    """With a budget that holds one large request and a few small ones, a large
    request waiting at the head of the queue is passed by small ones (a bounded
    number of times) and still completes."""
    big = WL.served_requests(1, seed=31, paths=(20000, 20001), nv_max=1024, nl_max=256)[0]
    big["args"][4] = WL.cap_dirs(200, 10.0, +1.0, np.random.default_rng(1))
    big["args"][5] = WL.cap_dirs(900, 10.0, -1.0, np.random.default_rng(2))
    small = WL.served_requests(12, seed=32, paths=(500, 2000), nv_max=16, nl_max=8)
    with Server(slots=1) as srv:  # the reservation of each request alone
        est_big = srv.wait(srv.submit_field(holder(big)))[1]["reserved_bytes"]
        est_small = max(srv.wait(srv.submit_field(holder(r)))[1]["reserved_bytes"] for r in small)
    budget = est_big + 3 * est_small
    with Server(slots=3, hbm_budget=budget) as srv:
        first = srv.submit_field(holder(big))      # occupies most of the budget
        t_big = srv.submit_field(holder(big))      # does not fit beside the first
        ts = [srv.submit_field(holder(r)) for r in small]
        res_small = [srv.wait(t) for t in ts]
        u_big, info_big = srv.wait(t_big)
        srv.wait(first)
    assert any(info["start_ms"] < info_big["start_ms"] for _, info in res_small)
    for r, (u, _) in zip(small, res_small):
        assert rel(u, MC.field_from_args(holder(r))) < SAME_TOL_MIXED
    assert rel(u_big, MC.field_from_args(holder(big))) < SAME_TOL_MIXED_LARGE
