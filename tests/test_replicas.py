"""Trial replicas over two processes (gloo on the CPU).

The multi-GPU path has no collective on the data path: each rank runs its
contiguous share of the trials and rank 0 gathers the per-trial results.
This test runs that host logic with two gloo ranks, the oracle standing in
for each rank's engine, and checks that the gathered results equal a single
process's, trial by trial and in order.
"""

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
N, E, STEPS = 1200, 1200 * 60, 80


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _trial_counts(spec):
    import fis.connectome as C
    from oracle import oracle as O

    c = C.synthetic(n=N, e=E, seed=2, cache=False).without(spec.silenced)
    o = O.Oracle.from_connectome(c, batch=1, no_refractory=spec.stim, seed=spec.seed,
                                 streams=[0])
    o.rates[0, np.asarray(spec.stim)] = np.float32(spec.rate_hz)
    raster = o.run(spec.steps, raster=True)
    return np.unpackbits(raster[:, 0], axis=1, bitorder="little")[:, :N].sum(0)


def _specs():
    from fis.batch import random_specs

    return random_specs(N, 5, 99, STEPS, stim_range=(100, 300), silenced_range=(1, 20))


def _rank_main(rank, world, port, out_path):
    for p in (ROOT / "fly-in-silico_b200", ROOT):
        sys.path.insert(0, str(p))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    from fis.replicas import gather_results, shard

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    mine, offset = shard(_specs(), world, rank)
    local = (offset, [_trial_counts(s) for s in mine])
    merged = gather_results(local, world, rank)
    if rank == 0:
        np.save(out_path, np.stack(merged))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_is_contiguous_and_complete():
    from fis.replicas import shard

    items = list(range(11))
    parts = [shard(items, 4, r) for r in range(4)]
    assert [p[1] for p in parts] == [0, 3, 6, 9]
    assert sum((p[0] for p in parts), []) == items


@pytest.mark.timeout(300)
def test_two_gloo_ranks_gather_equals_single_process(tmp_path):
    import torch.multiprocessing as mp

    out = tmp_path / "gathered.npy"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2,
                       start_method="spawn", join=True)
    got = np.load(out)
    want = np.stack([_trial_counts(s) for s in _specs()])
    assert got.shape == (5, N)
    assert np.array_equal(got, want)
