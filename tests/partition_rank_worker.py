"""One rank of a line-partitioned solve launched by torchrun (the launch
bench.py --gpus N uses): RANK / WORLD_SIZE / MASTER_* from the environment,
gloo process group, the partition's sweeps by the oracle (tests/
test_partition_cpu.OracleSweeper), the halo exchange by DistExchange on host
buffers.  Writes its owned cells' U, the sweep count and the global norm
history to <out>/rank<r>.npz.  Used by tests/test_partition_cpu.py."""
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)


def main(out_dir, lens, seed, tol):
    import torch.distributed as dist

    from test_partition_cpu import OracleSweeper, _problem
    from triblocksolve_b200.partition import DistExchange, PartitionedSolve, partition_lines
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        mesh, jac = _problem(lens, seed)
        part = partition_lines(mesh, world)[rank]
        s = OracleSweeper(part, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs)
        n, hist = PartitionedSolve([s], DistExchange(part, s, device="cpu")).solve(tol, 40)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), n=n, hist=hist,
                 U=s.base.U[:part.nelem_own * 9], elems=part.elems[:part.nelem_own])
        dist.barrier()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1], [int(x) for x in sys.argv[2].split(",")], int(sys.argv[3]),
         float(sys.argv[4]))
