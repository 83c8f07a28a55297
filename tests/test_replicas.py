"""The multi-process path of bench.py on CPU (world size 2, gloo).

`bench.py --gpus N` runs N independent replicas of the workload (rays are
independent; no collective on the data path).  The replicas' plumbing --
process group, per-rank seeds, a barrier before each timed region, the
slowest rank's time and the sum of the work -- lives in rt_b200/replicas.py
and is exercised here with two gloo ranks; the reference arm under torchrun
prints one line from rank 0 while the other rank exits without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from rt_b200 import replicas
    w, r, _ = replicas.init("gloo", timeout_s=60)
    res = {"world": w, "rank": r, "seed": replicas.seed(1000, r)}
    replicas.barrier()
    res["max"] = replicas.max_over_ranks(1.5 * (r + 1), device="cpu")   # device times 1.5, 3.0 ms
    res["sum"] = replicas.sum_over_ranks(10 * (r + 1), device="cpu")    # work 10 + 20
    replicas.finish()
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(res, f)


def test_replica_reductions_with_two_gloo_ranks(tmp_path):
    port = free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [x["rank"] for x in res] == [0, 1] and all(x["world"] == 2 for x in res)
    assert res[0]["seed"] != res[1]["seed"]                 # every replica traces its own rays
    assert all(x["max"] == 3.0 for x in res)                 # the job's time is the slowest rank's
    assert all(x["sum"] == 30.0 for x in res)                # the job's work is every rank's


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    from rt_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    assert replicas.init("gloo") == (1, 0, 0)
    assert replicas.max_over_ranks(2.5, device="cpu") == 2.5
    assert replicas.sum_over_ranks(7, device="cpu") == 7.0
    replicas.barrier()
    replicas.finish()


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_two_ranks():
    """Rank 0 times the CPU reference path and prints one JSON line; rank 1
    exits 0 without work."""
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=550, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    # the same workload config as the GPU arm's line (bench.workload_config)
    sys.path.insert(0, ROOT)
    import bench
    from rt_b200 import schemes as S
    beams = S.c1_beams()
    assert d["config"] == bench.workload_config(S.total_rays(beams), len(beams))
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
