"""The multi-rank (replicas) plumbing of bench.py, as two gloo processes on CPU.

Multi-GPU runs are independent replicas: each rank solves its own instance and the ranks only
meet for the barrier around the timed region and the max over ranks of the device time.  This
runs that plumbing with world size 2 on the CPU (backend gloo): the rendezvous on 127.0.0.1,
the barrier, the max over ranks, and the reference arm's rule that only rank 0 works and
prints while the other ranks return 0 without output.
"""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout
from types import SimpleNamespace

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      SDPX_B200_DIST_BACKEND="gloo")
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup()
    res = {"world": w, "rank": r, "local": local, "backend": dist.get_backend()}
    bench.barrier(w)
    res["max"] = bench.max_over_ranks(w, 10.0 + r)
    if r != 0:  # the reference arm on a rank other than 0: no work, no output, exit code 0
        buf = io.StringIO()
        with redirect_stdout(buf):
            rc = bench.run_reference(SimpleNamespace(steps=1, warmup=0, gpus=w), w, r)
        res["ref_rc"], res["ref_out"] = rc, buf.getvalue()
    bench.barrier(w)
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, x in enumerate(res):
        assert x["world"] == world and x["rank"] == r and x["local"] == r
        assert x["backend"] == "gloo"
        assert x["max"] == 10.0 + world - 1  # every rank sees the slowest rank's value
    assert res[1]["ref_rc"] == 0 and res[1]["ref_out"] == ""
