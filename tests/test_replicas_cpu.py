"""The multi-rank (replicas) path on CPU: two gloo ranks split a batch of
independent XXZ-field chains, solve their share with the oracle DMRG, and
rank 0 gathers the energies in chain order; the max-over-ranks time reduction
is checked too.  No GPU and no data-path collective are involved."""
import ast
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _chains(n):
    rng = np.random.default_rng(7)
    return [(6, list(rng.uniform(-0.1, 0.1, 6))) for _ in range(n)]


def _solve(item):
    from oracle import qdmrg
    L, h = item
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    H = qdmrg.QMPO(L, dh=h)
    return qdmrg.dmrg(psi, H, 3, [16], [1e-12], [4])


def _worker(rank, world, port, out_path):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tensor-tools_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    from tt_b200 import replicas
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        energies = replicas.run_chains(_chains(5), _solve)
        tmax = replicas.max_over_ranks(float(rank + 1))
        if rank == 0:
            with open(out_path, "w") as f:
                f.write(repr((energies, tmax)))
    finally:
        dist.destroy_process_group()


def test_partition_is_balanced_and_contiguous():
    from tt_b200 import replicas
    for n in (0, 1, 5, 64):
        for w in (1, 2, 3, 8):
            parts = [replicas.partition(n, w, r) for r in range(w)]
            assert [i for p in parts for i in p] == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_split_chains(tmp_path):
    out = tmp_path / "res.txt"
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(out)), nprocs=2, join=True, start_method="spawn")
    energies, tmax = ast.literal_eval(out.read_text())
    ref = [_solve(c) for c in _chains(5)]
    assert len(energies) == 5
    np.testing.assert_allclose(energies, ref, rtol=0, atol=1e-12)
    assert tmax == 2.0
