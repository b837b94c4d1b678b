"""The replica plumbing of the bench (barrier, max over ranks, whole-job
rate) with world_size 2 on the gloo backend, CPU only."""
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
    replicas.barrier()
    with open(f"{out}.{rank}", "w") as f:
        json.dump({"ws": replicas.replica_env()[0], "max": mx, "rate": rate}, f)
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


def test_single_process_is_a_no_op(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from diffmom_b200 import replicas
    replicas.init("gloo")
    replicas.barrier()
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(10, 1000.0) == 10.0
    replicas.finalize()
