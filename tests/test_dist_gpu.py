"""dist.halo_product on the GPU with a one-rank NCCL group (the GPU steps:
getmct, shrink_col, the product over the compact P), in a spawned child so
the process group does not outlive the test. The multi-rank exchange itself
is covered by the gloo tests on the CPU."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _child(rank, port, out_dir):
    import torch
    import torch.distributed as dist
    import nsp_b200 as nb
    import oracle
    from nsp_b200 import dist as nd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        A = nb.gen.random(3000, 2000, 0, 20, seed=5)
        P = nb.gen.random(2000, 1500, 0, 9, seed=6)
        C = nd.halo_product(A.to_device(), P.to_device(), nd.row_offsets(2000, 1), 0).to_host()
        rp, col, val = oracle.spgemm(A, P)
        assert np.array_equal(C.rowptr, rp) and np.array_equal(C.col, col)
        assert np.array_equal(C.val, val)
        open(os.path.join(out_dir, "ok"), "w").close()
    finally:
        dist.destroy_process_group()


def test_halo_product_one_rank(cuda, tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_child, args=(_free_port(), str(tmp_path)), nprocs=1,
                       start_method="spawn", join=True)
    assert os.listdir(tmp_path) == ["ok"]
