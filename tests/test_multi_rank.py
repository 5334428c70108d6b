"""The N > 1 paths of bench.py, as two gloo ranks on CPU.

The march path does not shard: N GPUs run N independent replicas, each
marching its own view, with no collective on the data path.  What the ranks
share is bookkeeping: a barrier around the timed region, the maximum of the
ranks' times, and the whole-job rate (all ranks' rays over the slowest rank's
time).  The reference arm runs on rank 0 only; the other ranks exit 0."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    w, r, local, dist = bench.dist_setup()
    try:
        # rank k's device time is 1 + k seconds: the job is as slow as rank 1
        rate = bench.job_mrays(dist, w, 1_000_000, 4, 1.0 + r)
        bench.barrier(dist)
        cam = bench.camera_for(bench.scenes.SCENE_LARGE, 64, 48, r)
        with open(os.path.join(out_dir, f"r{r}.json"), "w") as f:
            json.dump({"rank": r, "world": w, "local": local, "rate": rate, "cam": list(cam.position)}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_replica_bookkeeping_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    res = [json.load(open(tmp_path / f"r{k}.json")) for k in range(2)]
    assert [r["rank"] for r in res] == [0, 1] and all(r["world"] == 2 for r in res)
    # 2 ranks x 1M rays x 4 steps over the slower rank's 2 s
    assert all(r["rate"] == pytest.approx(4.0) for r in res)
    assert res[0]["cam"] != res[1]["cam"], "each replica marches its own view"


@pytest.mark.timeout(300)
def test_reference_arm_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--scene", "small", "--width", "64", "--height", "48",
           "--steps", "1", "--warmup", "0", "--cpu-rows", "8"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, "rank 0 alone prints the reference line"
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
