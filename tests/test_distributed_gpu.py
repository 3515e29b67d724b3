"""GPU, two ranks: render_sharded and adjoint_sharded through real Plans. Both ranks run on one GPU
as separate processes, each tracing its own photon range with its own kernels (no kernel waits on
the other rank); the films and gradients are summed over gloo on the host. The result must equal
the single-process render and gradient of the same photons."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import simpler_b200 as sb
from simpler_b200 import _lib as L

pytestmark = pytest.mark.gpu

N = 200_001                                   # not a multiple of the world size


def _setup():
    return sb.config_planewave(seed=13, spatial_x=32, spatial_y=32, path_length_bins=8, precision_mode=L.PREC_MIXED)


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def all_reduce(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        dist.all_reduce(t)
        return t.numpy()

    plan = sb.Plan(_setup())
    film, counts = sb.render_sharded(plan, N, rank, world, all_reduce)
    G = sb.roi_weights(plan.setup, 16)
    grad, acounts = sb.adjoint_sharded(plan, G, N, rank, world, all_reduce)
    plan.close()
    if rank == 0:
        np.savez(out, film=film, photons=counts["photons"], grad=grad, adj_photons=acounts["photons"])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_render_and_adjoint_match_single_process(tmp_path):
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "shard.npz")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = np.load(out)
    s = _setup()
    single, st = sb.render(s, N)
    assert int(res["photons"]) == N == st.photons
    # FP64 films: the sum of the two shards differs from one render by the order of the atomics
    assert np.abs(res["film"] - single).sum() <= 1e-12 * np.abs(single).sum()
    plan = sb.Plan(s)
    g1, _ = plan.adjoint(sb.roi_weights(s, 16), 0, N, N)
    plan.close()
    assert int(res["adj_photons"]) == N
    np.testing.assert_allclose(res["grad"], g1, rtol=1e-6)
