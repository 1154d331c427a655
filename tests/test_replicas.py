"""The N > 1 path on the host: one process per GPU as torchrun starts them,
here as world-size-2 gloo groups on the CPU (replicas only: no collective on
the data path, a start barrier and the max over ranks of the timed interval)."""
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
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world)})
    sys.path.insert(0, ROOT)
    from emergence_b200 import replicas
    w, r, local = replicas.init_from_env("gloo", timeout_s=60)
    replicas.barrier(w)
    # each rank "timed" a different interval; all must agree on the slowest
    ms = replicas.max_over_ranks(10.0 * (rank + 1), w, device="cpu")
    rate = replicas.whole_job_rate(1000, w, ms)
    replicas.finish(w)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"world": w, "rank": r, "local": local, "ms": ms, "rate": rate}, f)


def test_max_over_ranks_with_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, g in enumerate(got):
        assert (g["world"], g["rank"], g["local"]) == (world, r, r)
        assert g["ms"] == 20.0  # the slower rank's time, on every rank
        assert g["rate"] == pytest.approx(1000 * world / 0.020)


def test_single_process_needs_no_group(monkeypatch):
    sys.path.insert(0, ROOT)
    from emergence_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.init_from_env("gloo") == (1, 0, 0)
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    replicas.barrier(1)
    replicas.finish(1)


def test_reference_arm_under_torchrun_prints_one_line():
    """bench.py --impl reference launched like the two-GPU run: rank 0 times
    the CPU reference and prints the only JSON line; rank 1 exits 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--grid", "48"]  # a small grid: the default is the full 256^3 workload
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env={**os.environ, "OMP_NUM_THREADS": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
