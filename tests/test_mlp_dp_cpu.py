"""CPU (gloo, world size 2): data-parallel gradient averaging of the learned initialiser's MLP.

Each rank computes the oracle's gradient of its shard (shards of different
sizes); data_parallel_gradients must return the full-batch gradient and loss
on both ranks. The GPU path (TileMLP.data_parallel_step) uses the same
function with the tensor-core gradients and NCCL.
"""
import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

D, H, O = 128, 128, 13


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from complex_valued_quadratic_phase_gaussian_b200.mlp import data_parallel_gradients
        from oracle import mlp as om
        rng = np.random.default_rng(0)
        X = rng.normal(size=(20, D))
        T = rng.normal(size=(20, O))
        wout = np.ones(O)
        w = om.init_weights(D, H, O, seed=1).astype(np.float64)
        lo, hi = (0, 7) if rank == 0 else (7, 20)
        fn = lambda: tuple(torch.as_tensor(a, dtype=torch.float64) for a in om.forward_backward(w, X[lo:hi], T[lo:hi], wout, D, H, O,
                                                                         rounding=False)[::2])
        loss, g = data_parallel_gradients(fn, hi - lo)
        full_loss, _, full_g = om.forward_backward(w, X, T, wout, D, H, O, rounding=False)
        q.put((rank, float(abs(loss.item() - full_loss) / full_loss),
               float(np.linalg.norm(g.numpy() - full_g) / np.linalg.norm(full_g))))
    finally:
        dist.destroy_process_group()


def test_data_parallel_gradients_equal_full_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, dl, dg in res:
        assert dl < 1e-12 and dg < 1e-12, (rank, dl, dg)
