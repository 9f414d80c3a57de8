"""The benchmark's N-rank path on CPU: world size 2 over gloo.  Each rank
solves its own shard of the workload (per-cell solves are independent, so no
collective touches the data); the ranks only agree on the slowest rank's time.
The per-cell solve runs on the oracle here, standing in for the GPU."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

pytestmark = pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, cells, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        cfg, mech, inputs = bench.workload("c210_uneven", cells, rank)
        R = oracle.Restatement(mech, tableau_kind=cfg["stages"])
        y, stats = R.solve_per_cell(inputs, cfg["dt"], threads=1)
        # a deliberately uneven per-rank time: the job time must be the maximum
        seconds = 1.0 + rank
        (job_seconds,) = bench.max_over_ranks([seconds], dist, "cpu")
        value = bench.job_throughput(cells, world, 1, job_seconds)
        digest = torch.tensor([float(inputs["temperature"].sum())], dtype=torch.float64)
        gathered = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, digest)
        np.savez(f"{out_path}.{rank}.npz", y=y, accepted=stats[:, 3], job_seconds=job_seconds, value=value,
                 digests=np.array([g.item() for g in gathered]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_solve_disjoint_shards_and_agree_on_time(tmp_path):
    world, cells = 2, 8
    out = str(tmp_path / "rank")
    mp.start_processes(_rank_main, args=(world, _free_port(), cells, out), nprocs=world, start_method="spawn")
    r0, r1 = (np.load(f"{out}.{r}.npz") for r in range(world))
    # shards are different inputs (seeded per rank) ...
    assert r0["digests"][0] != r0["digests"][1]
    np.testing.assert_array_equal(r0["digests"], r1["digests"])
    # ... every rank agreed on the slowest rank's time, and the job value counts all ranks' cells
    assert float(r0["job_seconds"]) == float(r1["job_seconds"]) == 2.0
    assert float(r0["value"]) == float(r1["value"]) == cells * world / 2.0
    # and each shard's solve equals the same cells solved by a single process
    import bench
    for rank, r in enumerate((r0, r1)):
        cfg, mech, inputs = bench.workload("c210_uneven", cells, rank)
        R = oracle.Restatement(mech, tableau_kind=cfg["stages"])
        y, stats = R.solve_per_cell(inputs, cfg["dt"], threads=1)
        np.testing.assert_array_equal(r["y"], y)
        np.testing.assert_array_equal(r["accepted"], stats[:, 3])
