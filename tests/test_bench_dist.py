"""The multi-rank host logic of bench.py on CPU: world size 2 over gloo.

A single text does not shard, so N ranks build N independent replicas (or N independent batches and
request streams); the process group only carries the barriers and the max/sum of per-rank results.
These tests run that plumbing with two CPU processes, no GPU.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world), "SADCS_DIST_BACKEND": "gloo"})
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist

    w, r, local = bench.dist_setup(world)
    try:
        bench.barrier(w)
        result = {
            "world": w, "rank": r, "local": local,
            # a slower rank 1: the job's time is the max over ranks
            "max": bench.max_over_ranks(10.0 + 5.0 * r, w),
            # each rank processed its own text of (r + 1) MiB
            "sum": bench.sum_over_ranks(float((r + 1) << 20), w),
            "seed": bench.rank_seed(4, r),
            "share": bench.batch_share(64, w, r),
        }
        bench.barrier(w)
    finally:
        dist.destroy_process_group()
    Path(out_dir, f"rank{r}.json").write_text(json.dumps(result))


def test_two_ranks_reduce_and_seed(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn", join=True)
    results = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, res in enumerate(results):
        assert (res["world"], res["rank"], res["local"]) == (2, r, r)
        assert res["max"] == 15.0
        assert res["sum"] == float(3 << 20)
    # every rank builds its own synthetic batch / request stream
    assert results[0]["seed"] != results[1]["seed"]
    assert results[0]["seed"] == 4  # rank 0 keeps the single-GPU workload
    # one batch of 128 texts split across the two ranks: every text once, loads balanced
    from sadcs_b200 import workloads as W

    shares = [res["share"] for res in results]
    assert sorted(shares[0] + shares[1]) == list(range(128))
    lengths = W.batch_lengths(128, lo=1 << 10, hi=4 << 20, seed=4)
    loads = [int(sum(lengths[i] for i in share)) for share in shares]
    assert abs(loads[0] - loads[1]) <= int(lengths.max())


def test_partition_by_footprint():
    from sadcs_b200 import workloads as W

    lengths = [5, 1, 9, 3, 3, 7, 2, 8]
    parts = W.partition_by_footprint(lengths, 3)
    assert sorted(sum(parts, [])) == list(range(8))
    assert all(p == sorted(p) for p in parts)
    loads = sorted(sum(lengths[i] for i in p) for p in parts)
    assert loads == [12, 13, 13]  # longest first onto the least-loaded part
    assert W.partition_by_footprint(lengths, 1) == [list(range(8))]
    # a subset of a batch is generated identically on its own
    full = W.batch_texts(9, lo=1 << 10, hi=1 << 12, seed=4)
    part = W.batch_texts(9, lo=1 << 10, hi=1 << 12, seed=4, indices=[7, 2])
    assert (part[0] == full[7]).all() and (part[1] == full[2]).all()


def test_reference_arm_other_ranks_exit_without_work():
    """--impl reference under a launcher: rank 1 prints nothing, does no work, exits 0, joins no group."""
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                           "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert proc.returncode == 0, proc.stderr
    assert proc.stdout.strip() == ""


@pytest.mark.parametrize("workload", ["batch4096", "serve"])
def test_reference_arm_unavailable_lines(workload):
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", workload],
                          capture_output=True, text=True, timeout=120)
    assert proc.returncode == 0, proc.stderr
    line = json.loads(proc.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_gpus_flag_must_match_the_launcher():
    """--gpus N with a launcher that started another number of ranks is refused (exit 2), rather
    than running fewer replicas than asked and reporting them as N."""
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="1")
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                           "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert proc.returncode == 2
    assert "--gpus 2" in proc.stderr


def test_gpus_flag_without_a_launcher_starts_the_ranks():
    """--gpus 2 with no launcher starts two ranks itself; the reference arm's rank 0 prints the one
    line and rank 1 exits without work."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                           "--workload", "uniform8m", "--steps", "1", "--warmup", "0", "--reference-sample-mib", "1"],
                          env=env, capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [json.loads(x) for x in proc.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference"
    sys.path.insert(0, str(ROOT))
    import bench

    # the reference arm's config is the one this library's arm reports for the same workload
    assert lines[0]["config"] == bench.workload_config("uniform8m", 8 << 20, 1)
    assert lines[0]["cpu_baseline"]["sample"].startswith("first 1 MiB")
