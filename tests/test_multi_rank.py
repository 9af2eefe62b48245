"""Event sharding across ranks on CPU: two `gloo` ranks (one process each, as one process
per GPU) exercise the host logic of the multi-GPU path. Each rank reconstructs its own
share of the events with the oracle, the only collectives are scalar reductions, and the
reference arm of bench.py under torchrun prints exactly one line from rank 0."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_partitions_exactly():
    sys.path.insert(0, str(ROOT / "cms-julia_b200"))
    from pixeltrack.dist import rank_seed, shard
    for n in (0, 1, 7, 1000, 4097):
        for world in (1, 2, 3, 8):
            parts = [shard(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    assert len({rank_seed(5, r) for r in range(8)}) == 8


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cms-julia_b200"))
    import torch.distributed as dist

    from oracle import oracle
    from pixeltrack import dist as pdist
    from pixeltrack import gen
    assert pdist.init("gloo", timeout_s=60)
    conds = gen.conditions()
    blob, offs = gen.events(6, gen.MODE_PU, pu=10.0, seed=17)  # the same event list on every rank
    lo, hi = pdist.shard(6, world, rank)
    orc = oracle.Oracle(conds)
    hits = 0
    for e in range(lo, hi):
        orc.run_event(bytes(blob[offs[e]:offs[e + 1]]), 63)
        hits += orc.counts()["n_hits"]
    total = pdist.sum_over_ranks(hits)
    slowest = pdist.max_over_ranks(float(rank + 1))
    (Path(out_dir) / f"rank{rank}.json").write_text(json.dumps({"hits": hits, "total": total, "max": slowest}))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_share_the_events(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cms-julia_b200"))
    from oracle import oracle
    from pixeltrack import gen
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    conds = gen.conditions()
    blob, offs = gen.events(6, gen.MODE_PU, pu=10.0, seed=17)
    orc = oracle.Oracle(conds)
    single = 0
    for e in range(6):
        orc.run_event(bytes(blob[offs[e]:offs[e + 1]]), 63)
        single += orc.counts()["n_hits"]
    assert res[0]["total"] == res[1]["total"] == single == res[0]["hits"] + res[1]["hits"]
    assert res[0]["max"] == res[1]["max"] == 2.0


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--events", "8", "--cpu-sample", "8", "--pu", "10"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
