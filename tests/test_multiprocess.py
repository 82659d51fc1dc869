"""CPU, world size 2 over gloo: column sharding of the evaluation gives the same Y as one
process (the compute per rank is the oracle here; on GPUs it is the CUDA evaluator)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from matrox_ru_b200.shard import column_range


def test_column_range_partitions():
    for r in (0, 1, 5, 64, 1023):
        for world in (1, 2, 3, 8):
            spans = [column_range(r, k, world) for k in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == r
            assert all(spans[k][1] == spans[k + 1][0] for k in range(world - 1))
            widths = [b - a for a, b in spans]
            assert max(widths) - min(widths) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, path, out_dir):
    import torch
    import torch.distributed as dist
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import oracle as O
    from matrox_ru_b200 import structure as S
    from matrox_ru_b200.shard import sharded_apply
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cds = S.CDS.load(path)

    def local(Wslab):
        r = Wslab.shape[1]
        TW = cds.to_tree_order(Wslab.numpy())
        return torch.as_tensor(cds.from_tree_order(O.eval_h2b(cds, TW, r), r))

    W = torch.as_tensor(np.random.default_rng(0).standard_normal((cds.n, 13)))
    Y = sharded_apply(local, W)
    np.save(os.path.join(out_dir, f"y{rank}.npy"), Y.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo_match_single_process(tmp_path):
    from conftest import GOLDEN, rel_err
    import oracle as O
    from matrox_ru_b200 import structure as S
    path = os.path.join(GOLDEN, "h2b_n384.npz")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(k, 2, port, path, str(tmp_path))) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    cds = S.CDS.load(path)
    W = np.random.default_rng(0).standard_normal((cds.n, 13))
    want = cds.from_tree_order(O.eval_h2b(cds, cds.to_tree_order(W), 13), 13)
    for k in range(2):
        got = np.load(tmp_path / f"y{k}.npy")
        assert rel_err(got, want) <= 1e-13
