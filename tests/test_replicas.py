"""The multi-GPU form of the benchmark: one process per GPU, each evaluating
its own replica of the system (the MSM evaluation of one system is not
split across GPUs), timing reduced as the max over ranks and throughput
summed over ranks. These run the process-group plumbing of bench.py with
two gloo ranks on the CPU, and the reference arm under two ranks (rank 0
alone runs and prints; the other rank exits 0 without work).
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank) and pg is not None
    bench.barrier(pg)
    # per-rank step times: the job's step time is the slowest rank's
    ms = bench.reduce_max(pg, 2.0 + rank)
    value = 1000 * w / (ms * 1e-3)  # 1000 atoms per replica
    bench.barrier(pg)
    pg.destroy_process_group()
    with open(os.path.join(out, "rank%d.json" % rank), "w") as f:
        json.dump({"ms": ms, "value": value}, f)


def test_replica_timing_is_max_over_ranks(tmp_path):
    port = _free_port()
    tmp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    for rank in range(2):
        d = json.load(open(tmp_path / ("rank%d.json" % rank)))
        assert d["ms"] == 3.0
        assert d["value"] == pytest.approx(2 * 1000 / 3e-3)


def test_reference_arm_under_two_ranks():
    """One step of the reference arm (one FF_energy of the 1M-atom box on
    one host core, about a minute here) under two ranks."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=2", "--master-addr=127.0.0.1",
           "--master-port=%d" % _free_port(), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-procs", "1"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["cpu_baseline"]["cores"] == 1
    # the same workload as the GPU arm names
    import bench
    assert d["config"] == bench.WORKLOAD_CONFIG


def test_batch_cpu_reference_on_small_systems():
    """The batch section's CPU baseline: the reference's C code on a few small
    ion boxes of the batch workload, in independent spawned processes,
    every atom counted once."""
    sys.path.insert(0, ROOT)
    import bench
    from msmpb_b200 import systems
    from oracle.oracle import RefFF
    if not RefFF.available():
        pytest.skip("reference library not built (oracle/build_ref.py)")
    sysl = systems.ion_batch(6, seed=5, n_min=500, n_max=1500)
    out = bench.batch_cpu_reference(sysl, procs=3)
    assert out["value"] > 0 and out["kind"] == "reference"
    assert out["cores"] == min(3, os.cpu_count() or 1)
    atoms = sum(len(q) for q, _, _, _ in sysl)
    assert "all 6 systems (%d atoms)" % atoms in out["sample"]
