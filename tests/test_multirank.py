"""The N > 1 path of bench.py on CPU ranks (gloo, world size 2, 127.0.0.1).

Each rank segments its own volume (replicas, weak scaling, no data-path collective); the
step time is the max over ranks and the throughput counts every rank's voxels; the reference
arm runs on rank 0 only.  The GPU part of a rank is the single-GPU path the other tests cover.
"""
import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    c = bench.workload_case(size=24, seed=bench.replica_seed(rank), sweeps=3)
    # per-rank times differ; every rank must see the slowest one
    ms = bench.reduce_step_time(10.0 + 15.0 * rank, dist, "cpu")
    gvox = bench.whole_job_gvox(world, c.n, ms)
    # the reference arm does no work off rank 0
    ref = None
    if rank != 0:
        ref = bench.run_reference_arm(None, rank)
    res = {"rank": rank, "ms": ms, "gvox": gvox, "n": c.n, "shape": list(c.shape),
           "checksum": int(np.asarray(c.image, np.int64).sum()), "ref": ref}
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert all(r["ms"] == 25.0 for r in res)              # max over ranks
    n = res[0]["n"]
    assert all(r["n"] == n and r["shape"] == res[0]["shape"] for r in res)  # same work per rank
    assert res[0]["checksum"] != res[1]["checksum"]      # independent volumes
    assert res[0]["gvox"] == pytest.approx(world * n / 0.025 / 1e9)
    assert res[1]["ref"] is None


def test_bench_reads_the_committed_dram_traffic_table():
    """The roofline's `traffic` comes from the committed ncu summary: the headline OIFT
    launch's DRAM bytes are there, and they exceed its 12 B/voxel algorithmic bytes."""
    import bench
    t = bench.read_traffic("oift_persistent_kernel", "256^3")
    assert t is not None and t > 12 * 256 ** 3


def test_batch_cpu_baseline_runs_the_reference_on_host_processes():
    """The batch workload's cpu_baseline: each job of a small mix through the reference
    OIFT_Multi + ORelax_1_Multi in its own spawned process; the throughput is the jobs'
    count and voxels over the wall time."""
    import oracle as O
    if not O.ref_available():
        pytest.skip("reference library not built here")
    import bench
    from roift_b200 import synth
    jobs = []
    for seed in range(2):
        c = synth.small_case(seed=seed, shape=(12, 16, 20), pol=-0.3, adjacency=6, nlabels=1)
        jobs.append((c.image.reshape(-1), c.shape, c.seeds, c.seed_labels, c.pol, 5))
    sets_s, gvox_s, vox = bench.cpu_reference_batch(jobs, 2)
    assert vox == 2 * 12 * 16 * 20
    assert sets_s > 0 and gvox_s > 0
    assert abs(gvox_s / sets_s * 1e9 - vox / 2) < 1e-6 * vox
