"""The library's multi-GPU unit on one GPU: left-density shards (cl_compute_shard,
cl_request_create_shard) add up to the whole request in every form, and follow the dealing of
the plan's prepared densities; two gloo ranks (processes on the same GPU, no kernel waits on the
other rank) each compute their shard through the library and one all-reduce reproduces the
single-process integrals."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import coulombo_lattice_b200 as cl
from coulombo_lattice_b200 import multi, synth

from test_multi_gloo import density_shard_of_steps

pytestmark = pytest.mark.gpu

STEP = (synth.A_ZB / 4,) * 3


@pytest.mark.parametrize("mode", cl.ALL_MODES)
def test_shards_add_up_and_follow_the_dealing(mode):
    d = synth.build("c1", cells=(4, 4, 4))
    d["states"] = np.concatenate([d["states"], d["states"][:, :, ::-1]], axis=0)  # 8 states
    specs = cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 8, 4)
    with cl.CoulombCalculator(d["dims"], STEP, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 4)
        full = cc.compute(specs)
        for world in (2, 3, 50):
            parts = [cc.compute_shard(specs, r, world) for r in range(world)]
            assert np.abs(sum(parts) - full).max() <= 1e-12 * np.abs(full).max()
            owner = density_shard_of_steps([tuple(int(v) for v in s) for s in specs], 8, world)
            for r in range(world):
                assert np.all(parts[r][owner != r] == 0)
                assert np.allclose(parts[r][owner == r], full[owner == r], rtol=1e-12, atol=0)
            # prepared requests of the shards, replayed as one graph per shard
            reqs = [cc.request(specs, r, world) for r in range(world)]
            outs = []
            for rq in reqs:
                outs.append(rq.run().copy())
                rq.close()
            assert np.abs(sum(outs) - full).max() <= 1e-12 * np.abs(full).max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, mode, result_path):
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    d = synth.build("c1")
    specs = cl.enumerate_integrals("eeee,hhhh,ehhe,eheh", 4, 2)
    with cl.CoulombCalculator(d["dims"], STEP, mode) as cc:
        cc.initialize(dielectric=10.89)
        cc.set_states(d["states"], d["cells_idx"], 2)
        full = multi.compute_density_sharded(cc.compute_shard, specs)
        if rank == 0:
            np.save(result_path, np.stack([full, cc.compute(specs)]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("mode", [cl.MODE_FP64_SUBLATTICE, cl.MODE_FP32_SUBLATTICE])
def test_two_ranks_through_the_library(tmp_path, mode):
    out = str(tmp_path / "r.npy")
    mp.start_processes(_worker, args=(2, _free_port(), mode, out), nprocs=2, join=True, start_method="spawn")
    got, single = np.load(out)
    assert np.abs(got - single).max() <= 1e-12 * np.abs(single).max()
