"""k-hat sharding across ranks, on CPU with two gloo ranks.

Each rank computes its own directions (khat_shard) -- here with the oracle,
which stands in for a rank's GPU -- and rank 0 gathers the blocks; the
assembled spectrum must equal the single-process spectrum of all directions,
and the timing reduction must return the maximum over ranks.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gw_fopt_b200 import workloads as W
from gw_fopt_b200.sharding import khat_shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    from oracle import oracle as O
    from gw_fopt_b200.sharding import gather_spectra, khat_shard, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = W.config(1)
        kh = khat_shard(2, rank, world)
        local = O.compute_c_integral_khat(c.interior, c.exterior, kh, 12, 12, c.w[:8], 0.0, 1.5, 48,
                                          coefficients=c.coefficients, powers=c.powers, threads=1)
        full = gather_spectra(local, rank, world)
        mx = max_over_ranks(10.0 * (rank + 1))
        if rank == 0:
            np.savez(out_path, full=full, mx=mx)
    finally:
        dist.destroy_process_group()


def test_shards_are_disjoint_and_cover():
    world, k = 3, 5
    parts = [khat_shard(k, r, world) for r in range(world)]
    full = W.fibonacci_khat(k * world)
    assert all(p.shape == (k, 3) for p in parts)
    got = np.empty_like(full)
    for r, p in enumerate(parts):
        got[r::world] = p
    assert np.array_equal(got, full)
    with pytest.raises(ValueError):
        khat_shard(4, 2, 2)


def test_two_gloo_ranks_assemble_the_full_spectrum(tmp_path):
    from oracle import oracle as O
    world = 2
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    r = np.load(out)
    c = W.config(1)
    ref = O.compute_c_integral_khat(c.interior, c.exterior, W.fibonacci_khat(4), 12, 12, c.w[:8], 0.0, 1.5, 48,
                                    coefficients=c.coefficients, powers=c.powers, threads=1)
    assert r["full"].shape == ref.shape
    assert np.array_equal(r["full"], ref)
    assert float(r["mx"]) == 20.0
