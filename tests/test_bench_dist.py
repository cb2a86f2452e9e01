"""The benchmark's multi-process (replica) logic on CPU: two ranks with the
gloo backend, as `torchrun --nproc-per-node 2 bench.py` would start them on
GPUs with NCCL.  Checks the barrier, the max-over-ranks timing reduction and
that the reference arm runs and prints on rank 0 only."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path
from types import SimpleNamespace

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    r, w, _ = bench.dist_setup()
    assert (r, w) == (rank, world)
    bench.barrier(w)
    m = bench.max_over_ranks(float(rank + 1), w)
    args = SimpleNamespace(steps=1, warmup=0, nrhs=8, cpu_n=256, n=256, k=32, no_ref_gpu=True)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args, r, w)
    bench.barrier(w)
    dist.destroy_process_group()
    Path(outdir, f"rank{rank}.json").write_text(json.dumps({"max": m, "out": buf.getvalue()}))


def test_two_rank_replicas_gloo(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = [json.loads(Path(tmp_path, f"rank{r}.json").read_text()) for r in range(world)]
    assert all(x["max"] == float(world) for x in res)  # max over ranks of rank + 1
    assert res[1]["out"] == ""                          # only rank 0 prints
    line = json.loads(res[0]["out"].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == world
    assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
