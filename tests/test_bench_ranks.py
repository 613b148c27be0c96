"""The benchmark's multi-rank flow on CPU (gloo), its launcher, and the
checker-side input generator of the reference arm.

  - bench.timed_steps / job_rate / rank_seed, run by world-2 and world-3
    gloo ranks: every rank draws its own points, the job's time is the
    slowest rank's, and the whole-job rate counts every rank's points;
  - `bench.py --gpus 2` without a torchrun environment starts two ranks
    itself; rank 0 prints one line with n_gpus == 2 and the reference arm
    never maps the product library;
  - oracle/workload.py gives the same bits as the library's generator.
"""
import json
import os
import subprocess
import sys
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class SleepTimer:
    def start(self):
        self.t0 = time.perf_counter()

    def stop(self):
        self.t1 = time.perf_counter()

    def ms(self):
        return 1e3 * (self.t1 - self.t0)


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seed = bench.rank_seed(bench.SEED, rank)
        pts = bench.rank_seed(2, rank, 100)
        work = 0.02 * (rank + 1)  # rank r's step takes (r+1) x 20 ms

        def step():
            time.sleep(work)

        ms, ms_max = bench.timed_steps(step, 3, world, dist.barrier, SleepTimer())
        q.put((rank, seed, pts, ms, ms_max, bench.job_rate(1000, world, 3, ms_max)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rank_flow_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = [r[1] for r in res]
    assert seeds == [1 + r for r in range(world)] and len({r[2] for r in res}) == world
    slowest = max(r[3] for r in res)
    for rank, _, _, ms, ms_max, rate in res:
        assert ms_max == slowest  # every rank reports the slowest rank's time
        assert rate == pytest.approx(world * 1000 * 3 / (slowest / 1e3))
    assert slowest >= 3 * 20 * world * 0.9


def test_launcher_starts_n_ranks_and_reference_arm_skips_the_library(tmp_path):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    env["OMP_NUM_THREADS"] = "2"
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference", "--steps", "1",
           "--warmup", "0", "--points", "8192", "--cpu-seconds", "0.2"]
    r = subprocess.run(cmd, cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["config"]["d"] == 10 and line["config"]["num_subspaces"] == 92378
    assert not any("libsgb200" in lib for lib in line["libraries"]), line["libraries"]
    assert any("libasgb_ref" in lib for lib in line["libraries"])
    assert line["extrapolated_from_points"] <= 8192


def test_bench_rejects_a_world_size_mismatch():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "--gpus 2" in r.stderr


def test_checker_generator_matches_the_library_generator():
    from adaptive_sparse_grid_bench_b200 import inputs
    from oracle import workload
    for seed, count, start in ((1, 1000, 0), (7, 333, 12345), (0, 1, 1 << 40)):
        a = inputs.uniform01(seed, count, start)
        b = workload.uniform01(seed, count, start)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(inputs.uniform_points(1, 100, 10), workload.uniform_points(1, 100, 10))
    X = inputs.uniform_points(3, 50, 10).astype(np.float64)
    assert np.array_equal(inputs.f_gauss(X), workload.f_gauss(X))
