"""Replicas across ranks (pamtra_b200.replicas), world size 2 over gloo on
CPU: each rank computes its block of columns with the oracle, rank 0
gathers the blocks and finds the single-process result; the step time
reduces to the maximum over ranks.
"""
import os
import socket

import numpy as np
import pytest

from pamtra_b200 import replicas


def test_column_blocks_cover_once():
    for ncol in (1, 2, 7, 64, 4097):
        for world in (1, 2, 3, 8):
            blocks = [replicas.column_block(ncol, world, r) for r in range(world)]
            idx = np.concatenate([np.arange(ncol)[b] for b in blocks])
            assert np.array_equal(idx, np.arange(ncol))
            sizes = [len(range(ncol)[b]) for b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.column_block(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, result_file):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import datetime
    import torch.distributed as dist
    import oracle
    from pamtra_b200 import packing, workloads as wl
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pam = wl.c2_pam(5, seed=4)
        st = oracle.settings(packing.settings_from_nml(pam.nmlSet, 16))
        sp = packing.species_from_df(pam.df.data)
        cols = packing.profile_columns(pam.p, pam.df.nhydro)
        blk = replicas.slice_columns(cols, replicas.column_block(cols["ncol"], world, rank))
        tbs = []
        for c in range(blk["ncol"]):
            err, tb, _, _, _ = oracle.run_column(st, sp, blk, c, [89.0])
            assert err == 0
            tbs.append(tb)
        full = replicas.gather_blocks(np.stack(tbs))
        tmax = replicas.max_over_ranks(1.0 + rank)
        if rank == 0:
            np.save(result_file, full)
            with open(result_file + ".t", "w") as f:
                f.write(repr(tmax))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_gather_equals_single_process(tmp_path, oracle_mod):
    import torch.multiprocessing as mp
    from pamtra_b200 import packing, workloads as wl
    res = str(tmp_path / "tb.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), res), nprocs=2, join=True)
    got = np.load(res)
    pam = wl.c2_pam(5, seed=4)
    st = oracle_mod.settings(packing.settings_from_nml(pam.nmlSet, 16))
    sp = packing.species_from_df(pam.df.data)
    cols = packing.profile_columns(pam.p, pam.df.nhydro)
    ref = np.stack([oracle_mod.run_column(st, sp, cols, c, [89.0])[1] for c in range(5)])
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
    assert float(open(res + ".t").read()) == 2.0
