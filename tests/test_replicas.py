"""Replica bookkeeping for multi-GPU runs (rest_b200.replicas), on CPU with two
gloo ranks in spawned processes: the max / sum over ranks, balanced shards that
cover a set exactly once, and a sharded molecule set gathered on rank 0 in
input order (the SCF runner is a stand-in; no GPU is involved)."""
import json
import multiprocessing as mp
import os
import socket

import pytest

from rest_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r = replicas.init("gloo", timeout_s=60)
    res = {"max": replicas.max_over_ranks(r, 10.0 + rank), "sum": replicas.sum_over_ranks(r, 1.0 + rank),
           "shard": list(replicas.shard(11, r))}
    mols = [float(i) for i in range(11)]

    def runner(part):  # stand-in for run_molecule_set on this rank's GPU
        return [-m for m in part], [True] * len(part), [int(m) + 1 for m in part]

    res["set"] = replicas.run_set_sharded(r, mols, runner)
    replicas.barrier(r)
    replicas.finalize(r)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_single_process_needs_no_group():
    r = replicas.Ranks()
    assert not r.distributed
    assert replicas.max_over_ranks(r, 3.0) == 3.0
    assert list(replicas.shard(5, r)) == [0, 1, 2, 3, 4]
    assert replicas.gather_to_root(r, [1, 2]) == [1, 2]


@pytest.mark.parametrize("world", [2, 3])
def test_shards_are_balanced_and_cover_the_set(world):
    seen = []
    for rank in range(world):
        part = list(replicas.shard(11, replicas.Ranks(rank, world, rank, "gloo")))
        assert len(part) in (11 // world, 11 // world + 1)
        seen += part
    assert seen == list(range(11))


def test_two_gloo_ranks(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert res[0]["max"] == res[1]["max"] == 11.0
    assert res[0]["sum"] == res[1]["sum"] == 3.0
    assert res[0]["shard"] == [0, 1, 2, 3, 4, 5] and res[1]["shard"] == [6, 7, 8, 9, 10]
    assert res[1]["set"] is None
    assert res[0]["set"]["energies"] == [-float(i) for i in range(11)]
    assert res[0]["set"]["iterations"] == [i + 1 for i in range(11)]
    assert all(res[0]["set"]["converged"])
