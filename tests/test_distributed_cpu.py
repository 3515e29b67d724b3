"""CPU, two gloo ranks: the host logic of the multi-GPU decomposition -- each rank takes its own
contiguous photon range (shard_range) with streams keyed by the global photon index, then the FP64
films (or gradients, with their statistics) are summed -- reproduces the single-process result.
With no GPU here, the oracle traces each rank's range; tests/test_distributed_gpu.py runs the same
decomposition through real Plans on the GPU."""
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
    first, n = sb.shard_range(N, rank, world)
    _, img = ob.oracle_trace(_setup(), first, n, N, records=False, threads=2)
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


class _AdditivePlan:
    """Stands in for a Plan in the split-and-reduce logic: its 'gradient' of photons [first, first +
    n) is additive over photon ranges, as Plan.adjoint's is (tests/test_distributed_gpu.py runs the
    real Plans), and every call reports one dropped photon."""
    setup = sb.config_planewave()

    class _Stats:
        def __init__(self, n):
            self.photons, self.dropped, self.skipped, self.aborted, self.replay_mismatch = n, 1, 0, 0, 0

    def adjoint(self, G, first, n, weight):
        k = np.arange(first, first + n, dtype=np.float64)
        return np.array([k.sum(), (k * k).sum(), np.sin(k).sum(), float(n)]) / weight, self._Stats(n)


def _adjoint_rank(rank, world, port, out, n_photons):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def all_reduce(a):
        t = torch.from_numpy(a)
        dist.all_reduce(t)
        return t.numpy()

    g, counts = sb.adjoint_sharded(_AdditivePlan(), None, n_photons, rank, world, all_reduce)
    if rank == 0:
        np.save(out, np.concatenate([g, [counts["photons"], counts["dropped"]]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_adjoint_sharding_matches_single_process(tmp_path):
    n_photons = 1001                      # not a multiple of the world size
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "grad.npy")
    mp.spawn(_adjoint_rank, args=(2, port, out, n_photons), nprocs=2, join=True)
    sharded = np.load(out)
    single, counts = sb.adjoint_sharded(_AdditivePlan(), None, n_photons)
    assert np.allclose(sharded[:4], single, rtol=1e-12)
    assert single[3] * n_photons == n_photons          # every photon exactly once
    # the statistics travel with the gradient: photons counted once, drops from both ranks summed
    assert sharded[4] == n_photons == counts["photons"]
    assert sharded[5] == 2 * counts["dropped"] == 2
