"""The multi-GPU plumbing of the bench with world_size 2 on the gloo backend,
CPU only: barrier, max over ranks, whole-job rate, the partition of an
incidence sweep into disjoint shares and the gather of the per-incidence
results to rank 0."""
import json
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out):
    os.environ.update({"WORLD_SIZE": str(ws), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from diffmom_b200 import replicas
    replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    ms = 100.0 + 50.0 * rank          # rank 1 is the slower replica
    mx = replicas.max_over_ranks(ms)
    rate = replicas.aggregate_rate(1024, mx)
    # a sweep of 7 incidences: rank 0 takes 4, rank 1 takes 3; each "solves"
    # its share (sigma = incidence index + 0.5) and rank 0 gathers them all
    start, count = replicas.shard(7, ws, rank)
    sig = [i + 0.5 for i in range(start, start + count)]
    got = replicas.gather_to_rank0(sig)
    replicas.barrier()
    with open(f"{out}.{rank}", "w") as f:
        json.dump({"ws": replicas.replica_env()[0], "max": mx, "rate": rate, "share": [start, count],
                   "gathered": None if got is None else got.tolist()}, f)
    replicas.finalize()


def test_two_replicas_on_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(f"{out}.{r}")) for r in range(2)]
    for r in res:
        assert r["ws"] == 2
        assert r["max"] == 150.0                       # both ranks see the slower one
        assert r["rate"] == pytest.approx(2 * 1024 / 0.150)
    assert res[0]["share"] == [0, 4] and res[1]["share"] == [4, 3]
    assert res[0]["gathered"] == [i + 0.5 for i in range(7)]   # every incidence once, in order
    assert res[1]["gathered"] is None


def test_shard_partitions_every_unit_once():
    from diffmom_b200 import replicas
    for total in (0, 1, 7, 1024, 2048 + 3):
        for ws in (1, 2, 3, 8):
            seen = []
            for r in range(ws):
                a, n = replicas.shard(total, ws, r)
                seen.extend(range(a, a + n))
                assert n in (total // ws, total // ws + 1)
            assert seen == list(range(total))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_single_process_is_a_no_op(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from diffmom_b200 import replicas
    replicas.init("gloo")
    replicas.barrier()
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(10, 1000.0) == 10.0
    assert list(replicas.gather_to_rank0([1.0, 2.0])) == [1.0, 2.0]
    replicas.finalize()
