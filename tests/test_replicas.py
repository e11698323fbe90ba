"""Replica host logic (bench.py --gpus N) with two gloo ranks on the CPU.

Each rank advances its own lattice (the oracle stands in for the device
here) with its own noise seed; ranks meet only for the timing max and the
final gather of the plaquette series.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from prlgt2020_b200 import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w, r, _ = R.world_info()
        assert (w, r) == (world, rank)
        seed = R.replica_seed(7, r)
        o = O.Oracle((2, 2, 2, 2), 3)
        rng = O.Rand55(seed)
        for _ in range(2):  # the sweep measures the field it starts from
            obs = o.sweep(0.01, rng.gauss(o.V * 32))
        fake_seconds = 1.0 + r  # the slowest rank sets the job time
        tmax = R.max_over_ranks(fake_seconds)
        series = R.gather_series(obs.plaq.reshape(-1))
        rate = R.whole_job_rate(1.0, world, tmax)
        np.save(os.path.join(out_dir, "rank%d.npy" % r),
                np.array([seed, tmax, rate] + [x for s in series for x in s]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    a = np.load(tmp_path / "rank0.npy")
    b = np.load(tmp_path / "rank1.npy")
    assert a[0] != b[0]                      # distinct noise seeds
    assert a[1] == b[1] == 2.0               # max over ranks
    assert a[2] == b[2] == pytest.approx(1.0)  # 2 sweeps / 2 s
    assert np.array_equal(a[3:], b[3:])      # every rank gathered the same table
    half = (len(a) - 3) // 2
    assert not np.array_equal(a[3:3 + half], a[3 + half:])  # replicas differ


def test_single_process_fallbacks():
    assert R.max_over_ranks(3.5) == 3.5
    assert R.gather_series([1.0, 2.0]) == [[1.0, 2.0]]
    assert R.replica_seed(5, 0) == 5


def test_replica_seeds_of_nearby_jobs_do_not_collide():
    """Jobs whose base seeds are close (or c apart, for any small c) never
    give two (base, rank) pairs the same noise seed."""
    seen = {}
    for base in range(1000, 1064):
        for rank in range(16):
            s = R.replica_seed(base, rank)
            assert 0 <= s < 2 ** 64
            assert s not in seen, (base, rank, seen.get(s))
            seen[s] = (base, rank)
    assert R.replica_seed(1000 + 1000003, 0) != R.replica_seed(1000, 1)
    with pytest.raises(ValueError):
        R.whole_job_rate(1.0, 1, 0.0)
