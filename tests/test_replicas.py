"""The multi-GPU layer of the benchmark on CPU: replicas on gloo ranks.

The path does not shard (one system per replica), so N > 1 is N independent
replicas whose device times are combined as the maximum over ranks and whose
throughput adds up; only rank 0 of the reference arm does work.  These tests
run those pieces on world_size 2 with the gloo backend."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    ms = bench.job_time_ms(1.5 + rank, ws, device="cpu")
    v = bench.job_value(1000.0, ms, ws)
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"r{rank}.json").write_text(json.dumps({"ms": ms, "value": v}))


def test_job_time_is_max_over_ranks_and_value_adds_replicas(tmp_path):
    ws = 2
    mp.start_processes(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws,
                       start_method="spawn", join=True)
    r = [json.loads(Path(tmp_path, f"r{k}.json").read_text()) for k in range(ws)]
    assert r[0]["ms"] == r[1]["ms"] == 2.5
    assert r[0]["value"] == pytest.approx(2 * 1000.0 / 2.5e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(gpus=2, steps=1, warmup=0, impl="reference", seed=0)
    assert bench.reference_arm(args) == 0
    assert capsys.readouterr().out == ""
