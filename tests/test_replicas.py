"""The N > 1 path of bench.py on CPU: replicas with no data-path collective,
a barrier around the timed region and the maximum of the per-rank times
(world size 2, gloo), and the reference arm launched by torchrun (rank 0
alone runs and prints; the other ranks exit 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from edus_b200.replicas import ReplicaGroup, whole_job_rate

    g = ReplicaGroup("gloo", device="cpu", timeout_s=60)
    g.barrier()
    # per-rank "device times": rank 1 is the slower replica
    t = g.max(1.5 + rank)
    rate = whole_job_rate(g.world, units_per_step=1000, steps=4, max_seconds=t)
    g.barrier()
    g.close()
    with open(f"{out}.{rank}", "w") as f:
        json.dump({"rank": rank, "world": g.world, "max": t, "rate": rate}, f)


def test_replica_group_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    port = free_port()
    out = str(tmp_path / "r")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [json.load(open(f"{out}.{r}")) for r in range(2)]
    for r in res:
        assert r["world"] == 2
        assert r["max"] == 2.5  # both ranks see the slower rank's time
        assert r["rate"] == 2 * 1000 * 4 / 2.5  # whole-job units over the slowest rank's time


def test_replica_group_single_rank(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from edus_b200.replicas import ReplicaGroup

    g = ReplicaGroup("gloo", device="cpu")
    assert not g.active and g.max(3.0) == 3.0
    g.barrier()
    g.close()


def test_reference_arm_under_torchrun(tmp_path):
    """bench.py --impl reference launched like the 2-GPU run: one JSON line from rank 0, exit 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps",
           "1", "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["value"] == line["value"]
