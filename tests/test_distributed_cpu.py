"""CPU, two gloo ranks: the multi-GPU decomposition of bench.py -- each rank traces its own
contiguous photon range with streams keyed by the global photon index, then the FP64 films are
summed -- reproduces the single-process render. The oracle stands in for the per-rank kernel."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle_bridge as ob
import simpler_b200 as sb
from simpler_b200 import _lib as L

N = 1200


def _setup():
    return sb.config_plain_small(rng=L.RNG_PHILOX, seed=11, spatial_x=24, spatial_y=24, path_length_bins=6,
                                 precision_mode=L.PREC_MIXED)


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    per = N // world
    _, img = ob.oracle_trace(_setup(), rank * per, per, N, records=False, threads=2)
    t = torch.from_numpy(img)
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_photon_sharding_matches_single_process(tmp_path):
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "film.npy")
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    sharded = np.load(out)
    _, single = ob.oracle_trace(_setup(), 0, N, N, records=False, threads=2)
    assert np.allclose(sharded, single, rtol=1e-12, atol=1e-15)
