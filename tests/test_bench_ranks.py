"""The multi-process timing path of bench.py on the CPU: two ranks over the
gloo backend reach the barrier together and both get the slowest rank's
figures from the max-over-ranks reduction (what `bench.py --gpus N` does
with NCCL, one process per GPU)."""

import os
import socket
from datetime import timedelta

import numpy as np


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        import bench
        bench._barrier(world)
        vals = bench._max_over_ranks(world, [1.0 + rank, 10.0 - rank, -5.0 * rank])
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array(vals))
        bench._barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npy")
        np.testing.assert_array_equal(got, [2.0, 10.0, 0.0])


def test_single_process_is_identity():
    import bench
    assert bench._max_over_ranks(1, [np.float32(1.5), 2]) == [1.5, 2.0]
    bench._barrier(1)
