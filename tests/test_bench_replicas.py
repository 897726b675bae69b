"""The N > 1 plumbing of bench.py on CPU: two `gloo` ranks stand in for two
GPUs.  Each rank runs its own replica (no data-path collective); the
process group only brackets the timed region and takes the slowest rank's
time, and only rank 0 prints a line."""
import importlib.util
import io
import json
import os
import socket
import sys
import contextlib

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test",
                                                  os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    bench = _load_bench()
    rep = bench.Replicas("gloo", "cpu", timeout_s=60)
    res = {"rank": rep.rank, "world": rep.world}
    rep.barrier()
    # Uneven per-rank durations: rank r took (r + 1) * 0.5 s for 100 units.
    res["max"] = rep.max((rank + 1) * 0.5)
    res["rate"] = rep.rate(100.0, (rank + 1) * 0.5)
    res["sum"] = rep.sum(rank + 1)
    rep.close()
    # The reference arm runs on rank 0 alone: other ranks leave without work
    # and without printing.
    if rank != 0:
        buf = io.StringIO()
        args = type("A", (), {"workload": "fp64_8c_p3", "steps": 1, "warmup": 1,
                              "gpus": world})()
        with contextlib.redirect_stdout(buf):
            bench.run_reference(args)
        res["ref_stdout"] = buf.getvalue()
    out.put(res)


def test_replicas_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort(key=lambda r: r["rank"])
    for r in results:
        assert r["world"] == 2
        assert r["max"] == pytest.approx(1.0)
        # 200 units over the slowest rank's 1.0 s.
        assert r["rate"] == pytest.approx(200.0)
        assert r["sum"] == pytest.approx(3.0)
    assert results[1]["ref_stdout"] == ""


def test_replicas_single_rank_is_local(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    bench = _load_bench()
    rep = bench.Replicas("gloo", "cpu")
    assert rep.pg is None and rep.world == 1
    assert rep.max(2.5) == 2.5
    assert rep.rate(10.0, 2.0) == 5.0
    rep.close()


def test_bench_workloads_declared():
    bench = _load_bench()
    assert bench.WORKLOADS["fp64_32c_p7"][:4] == (32, 32, 32, 7)
    assert bench.stage_bytes_per_dof(False) == [40, 48, 48]
    assert bench.stage_bytes_per_dof(True) == [24, 28, 32]
    sys.argv = ["bench.py"]
    a = bench.parse()
    assert a.gpus == 1 and a.workload == "fp64_32c_p7" and a.impl == "ours"
