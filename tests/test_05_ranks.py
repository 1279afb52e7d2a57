"""The multi-GPU logic of bench.py on CPU ranks (gloo, world size 2): one
independent replica per rank (feram_mpi.F:33-36 runs one input per rank),
the device time as the maximum over ranks, the whole-job rate over all
ranks' sites; and the reference arm under torchrun, where rank 0 alone runs
and prints."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        w, r, loc = bench.rank_layout()
        ms = 10.0 + 5.0 * r  # this rank's device time
        m = bench.reduce_max(ms, w, dist, "cpu")
        v = bench.whole_job(4096, 100, m, w)
        cfg = bench.bench_config(16, 4096, w)
        with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
            json.dump({"layout": [w, r, loc], "seed": list(bench.replica_seed(r)), "max": m, "value": v,
                       "config": cfg}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time_and_sum_the_sites(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    r = [json.load(open(tmp_path / f"rank{i}.json")) for i in range(2)]
    assert [x["layout"] for x in r] == [[2, 0, 0], [2, 1, 1]]
    assert r[0]["seed"] != r[1]["seed"]                  # independent replicas
    assert r[0]["max"] == r[1]["max"] == 15.0            # the slowest rank's time on every rank
    assert r[0]["value"] == r[1]["value"] == 4096 * 100 * 2 / 15e-3
    assert r[0]["config"]["parallelism"] == "replicas x2"


def test_reference_arm_under_torchrun_prints_once(tmp_path):
    """bench.py --impl reference with two ranks: rank 0 times the oracle on
    a small sample and prints one line; rank 1 exits 0 without work; the
    product library is never loaded."""
    oracle_so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_so):
        pytest.skip("oracle not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "3",
           "--size", "16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["config"]["parallelism"] == "replicas x2"
    assert not any("libferam_gpu" in x for x in (d["repo_libs_loaded"] or []))
