"""The multi-process path on CPU: two gloo ranks, as torchrun would start
them, each reconstructing its own images with no exchange; only the timing
reductions are collective."""
import socket

import numpy as np
import torch.multiprocessing as mp

from jxr_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import jxr_b200 as J
    from tests._bridge import decode_synth
    r = replicas.init("gloo", timeout_s=60)
    # each replica decodes its own image (per-rank seed), as the benchmark's replicas do
    img = J.synth(64, 48, quality=70, overlap=2, seed=100 + rank, threads=1)
    out = J.OutputFormat(J.COLOR["RGB"], J.DEPTH["U8"], J.STORE["U8"], J.LAYOUT["RGB"], 64, 48)
    rc, pixels = decode_synth(img, out)
    r.barrier()
    result = dict(rank=rank, rc=rc, checksum=int(pixels.astype(np.int64).sum()), max=r.max(rank + 1.5),
                  sum=r.sum(rank + 1.0), shard=replicas.shard(list(range(7)), rank, world), backend=r.backend)
    r.close()
    queue.put(result)


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, queue)) for k in range(2)]
    for p in procs:
        p.start()
    results = sorted((queue.get(timeout=180) for _ in procs), key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [d["backend"] for d in results] == ["gloo", "gloo"]
    assert all(d["max"] == 2.5 and d["sum"] == 3.0 for d in results)
    assert sorted(results[0]["shard"] + results[1]["shard"]) == list(range(7))
    assert not set(results[0]["shard"]) & set(results[1]["shard"])
    # no exchange: each replica's result is what a single process computes
    import jxr_b200 as J
    from tests._bridge import decode_synth
    for d in results:
        assert d["rc"] == 0
        img = J.synth(64, 48, quality=70, overlap=2, seed=100 + d["rank"], threads=1)
        out = J.OutputFormat(J.COLOR["RGB"], J.DEPTH["U8"], J.STORE["U8"], J.LAYOUT["RGB"], 64, 48)
        rc, pixels = decode_synth(img, out)
        assert rc == 0 and int(pixels.astype(np.int64).sum()) == d["checksum"]


def test_single_replica_without_torchrun(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    r = replicas.init()
    assert (r.world, r.rank) == (1, 0)
    assert r.max(3.0) == 3.0 and r.sum(2.0) == 2.0
    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
