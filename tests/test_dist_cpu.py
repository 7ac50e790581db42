"""The multi-process host path of bench.py on CPU (gloo, world size 2).

With N GPUs every rank solves its own independent system (weak scaling):
the only collectives are the barrier and the max / sum of the per-rank
timings and sweep counts, which rank 0 turns into the whole-job value.
These tests run that aggregation with two gloo ranks, and the reference
arm under torchrun, where rank 0 alone works and prints.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE="2", LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local = bench.dist_env()
    d = bench.Dist(ws, r, local, "gloo")
    try:
        d.barrier()
        # per-rank: sweeps done and device milliseconds of its own system
        sweeps, ms = (80, 10.0) if rank == 0 else (72, 12.5)
        out[rank] = (d.reduce(ms, "max"), d.reduce(sweeps, "sum"), d.reduce(rank + 1, "max"))
        d.barrier()
    finally:
        d.close()


def test_gloo_aggregation_two_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(port, out), nprocs=2, join=True)
        res = dict(out)
    for rank in (0, 1):
        max_ms, all_sweeps, max_rank = res[rank]
        assert max_ms == 12.5 and all_sweeps == 152 and max_rank == 2
    # the whole-job value rank 0 reports: all ranks' sweeps over the slowest rank's time
    assert abs(152 / (12.5e-3) - 12160.0) < 1e-9


def test_aggregate_plain():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate([3.0, 7.5, 1.0], "max") == 7.5
    assert bench.aggregate([3, 4], "sum") == 7


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun_rank0_only():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--config", "c1", "--steps", "2", "--warmup", "1", "--gpus", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    import oracle
    # the reference's own kernels (oracle/_ref) where they were built, else the restatement
    assert line["cpu_baseline"]["kind"] == ("reference" if oracle.ref_available() else "port")


def test_reference_arm_does_not_load_the_product_library():
    """The CPU reference arm builds its system with the oracle's numpy
    generator: libtriblock.so must not be mapped in its process."""
    code = ("import sys, runpy\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--config', 'c1', '--steps', '1', "
            "'--warmup', '0']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit as e:\n    assert not e.code, e.code\n"
            "print('MAPS', 'libtriblock' in open('/proc/self/maps').read())\n")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "MAPS False" in p.stdout, p.stdout[-2000:]


def test_reference_byte_model():
    """bench.py's reference_model_gbs uses the reference's own byte count
    (src/main.cxx:146-175): 9.92 GB per sweep, 6.45 KB per cell, at
    1,200 x 1,280 cells with 9 x 9 blocks."""
    sys.path.insert(0, ROOT)
    import bench
    import triblocksolve_b200 as tbs
    m = tbs.Mesh.structured(1200, 1280)
    b = bench.reference_model_bytes(m)
    assert abs(b / 1e9 - 9.92) < 0.005
    assert 6440 < b / m.nelem < 6470
