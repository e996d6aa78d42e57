"""Multi-rank logic of the benchmark on CPU: two gloo ranks, one ensemble
member each.  Checks the barrier and max-over-ranks timing, the whole-job
aggregate, that members differ only by their seeded perturbation, and that
the reference arm runs on rank 0 only."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from cgd_b200 import physics as Ph
        r = bench.Ranks(rank, world, None)
        r.barrier()
        t = r.max(0.5 * (rank + 1))
        cfg = bench.member_config(Ph.CONFIGS["small"], rank)
        U = np.zeros((4, 8, 5), order="F")
        U[:, :, 0] = 1.0
        U[:, :, 4] = 300.0
        Ph.theta_noise(U, cfg.theta_noise, cfg.seed_theta)
        np.save(os.path.join(out, f"theta_{rank}.npy"), U[:, :, 4])
        with open(os.path.join(out, f"r{rank}.txt"), "w") as f:
            f.write(f"{t} {bench.aggregate(world, 10, t)} {cfg.seed_theta}")
        r.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    vals = [open(tmp_path / f"r{r}.txt").read().split() for r in range(2)]
    for t, agg, _ in vals:
        assert float(t) == 1.0               # max over ranks, seen by every rank
        assert float(agg) == 20.0            # 2 ranks x 10 steps / 1.0 s
    assert int(vals[1][2]) == int(vals[0][2]) + 1
    a, b = np.load(tmp_path / "theta_0.npy"), np.load(tmp_path / "theta_1.npy")
    assert not np.array_equal(a, b)
    assert np.abs(a - 300.0).max() <= 0.01 * 1.0001 and np.abs(b - 300.0).max() <= 0.01 * 1.0001


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import bench
    from cgd_b200 import physics as Ph

    class A:
        steps, warmup, gpus = 3, 1, 2
    bench.run_reference(A, Ph.CONFIGS["small"], rank=1)
    assert capsys.readouterr().out == ""


def test_single_rank_plumbing():
    import bench
    r = bench.Ranks(0, 1, None)
    r.barrier()
    assert r.max(2.5) == 2.5
    assert bench.aggregate(1, 100, 2.0) == 50.0


def test_reference_arm_line_on_rank_zero(capsys):
    """Rank 0 prints one JSON line with the contract's keys: the CPU
    restatement's rate as value, cpu_baseline describing the same run, and an
    e2e object with no host-device bytes (the CPU arm copies nothing)."""
    import json

    import bench
    from cgd_b200 import physics as Ph

    class A:
        steps, warmup, gpus = 1, 1, 1
    bench.run_reference(A, Ph.CONFIGS["small"], rank=0)
    lines = [l for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and abs(d["ms_per_step"] - 1e3 / d["value"]) <= 1e-6 * d["ms_per_step"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
