"""The multi-GPU path is replicas only: each rank samples its own shard with its own generator, no collective
on the data path.  Its host logic runs here on two `gloo` ranks on the CPU (no GPU): the shard ranges, the
per-rank seeds, MAX-over-ranks timing, the optional gather of every rank's occupations, and a rank that
fails before joining a collective (the others end with an error, they do not hang)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from photonic_engines_b200 import replicas as R


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_sampler(U, in_modes, shots, generator=None, **kw):
    """Stands in for fock_sample on the CPU: occupations [shots, m] whose rows carry the generator's draws."""
    m = U.shape[-1]
    occ = torch.zeros(shots, m, dtype=torch.int64)
    occ[:, 0] = torch.randint(0, 1000, (shots,), generator=generator)
    occ[:, 1] = len(in_modes)
    return occ


def _rank_main(rank, world, port, case, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    try:
        if case == "dies" and rank == 1:
            raise SystemExit(3)                      # never joins: rank 0's init or collective must time out
        R.init("gloo", timeout_s=10 if case == "dies" else 60)
        res = {}
        if case == "basic":
            res["shard"] = R.shard(11, world, rank)
            res["max"] = R.max_over_ranks(1.5 + rank)
            t = torch.full((3 + rank, 2), rank, dtype=torch.int64)
            res["gather"] = R.gather_rows(t).tolist()
            U = torch.zeros(4, 4)
            local = R.sample_replicas(U, [0, 1], 9, seed=5, sampler=_fake_sampler)
            res["local"] = local.tolist()
            res["all"] = R.sample_replicas(U, [0, 1], 9, seed=5, sampler=_fake_sampler, gather=True).tolist()
        elif case == "dies":
            try:
                R.max_over_ranks(1.0)
                res["error"] = None
            except Exception as e:                   # the collective's timeout, not a hang
                res["error"] = type(e).__name__
        out[rank] = res
        dist.barrier() if case == "basic" else None
        dist.destroy_process_group()
    except Exception as e:                           # rank 0 of the "dies" case may fail in init instead
        out[rank] = {"error": type(e).__name__, "where": "init"}


def _run(case, world=2):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, case, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        alive = [p for p in procs if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive, "a rank hung"
        return dict(out), [p.exitcode for p in procs]


def test_shards_cover_the_run_without_overlap():
    for total in (0, 1, 7, 2000, 2001):
        for W in (1, 2, 3, 8):
            ranges = [R.shard(total, W, r) for r in range(W)]
            assert ranges[0][0] == 0 and ranges[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        R.shard(10, 2, 2)


def test_replica_seeds_differ_per_rank():
    seeds = {R.replica_seed(7, r) for r in range(64)}
    assert len(seeds) == 64 and R.replica_seed(7, 3) == R.replica_seed(7, 3)


def test_single_process_is_a_plain_call():
    assert R.max_over_ranks(2.5) == 2.5
    t = torch.arange(6).reshape(3, 2)
    assert torch.equal(R.gather_rows(t), t)
    occ = R.sample_replicas(torch.zeros(3, 3), [0], 4, seed=1, sampler=_fake_sampler)
    assert occ.shape == (4, 3)


def test_two_gloo_ranks_shard_time_and_gather():
    out, codes = _run("basic")
    assert codes == [0, 0], (codes, out)
    assert [out[r]["shard"] for r in range(2)] == [(0, 6), (6, 11)]
    assert out[0]["max"] == out[1]["max"] == 2.5
    want = [[0, 0]] * 3 + [[1, 1]] * 4
    assert out[0]["gather"] == out[1]["gather"] == want
    assert len(out[0]["local"]) == 5 and len(out[1]["local"]) == 4          # 9 shots: 5 + 4
    assert out[0]["all"] == out[1]["all"] == out[0]["local"] + out[1]["local"]
    assert [r[0] for r in out[0]["local"][:4]] != [r[0] for r in out[1]["local"]]   # different generators


def test_a_rank_that_never_joins_ends_the_others_with_an_error():
    out, codes = _run("dies")
    assert codes[1] == 3
    assert out[0]["error"] is not None
