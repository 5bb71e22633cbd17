"""Multi-rank decomposition on CPU (gloo, world size 2): the round split and the left-density
split, each plus one all-reduce, reproduce the single-process integrals; structure partitioning
is balanced and complete."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from coulombo_lattice_b200 import multi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_path):
    import datetime
    import torch.distributed as dist
    from coulombo_lattice_b200 import synth
    from oracle import host as H
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    d = synth.build("c1", cells=(2, 2, 2))
    step = (synth.A_ZB / 4,) * 3
    specs = H.enumerate_integrals(H.Pattern("****", 2), 4)

    def partial(sp, mask):
        rounds = [k for k in range(8) if (mask >> k) & 1]
        return np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], step, sp,
                                            dielectric=10.89, rounds=rounds))

    full = multi.compute_sharded(partial, specs)
    if rank == 0:
        np.save(result_path, full)
    dist.barrier()
    dist.destroy_process_group()


def density_shard_of_steps(specs, n_inputs, world):
    """Shard of every integral in the library's dealing: the plan's prepared (left) densities in
    ascending product order, round-robin (restated here with the oracle's plan)."""
    from oracle import host as H
    plan = H.compute_plan([tuple(s) for s in specs], n_inputs * (n_inputs + 1) // 2)
    lefts = sorted({st[1][0] for st in plan})
    owner = {p: k % world for k, p in enumerate(lefts)}
    shard = np.zeros(len(specs), dtype=int)
    for (sid, left, _) in plan:
        shard[sid] = owner[left[0]]
    return shard


def _density_worker(rank, world, port, result_path):
    import datetime
    import torch.distributed as dist
    from coulombo_lattice_b200 import synth
    from oracle import host as H
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    d = synth.build("c1", cells=(2, 2, 2))
    step = (synth.A_ZB / 4,) * 3
    specs = H.enumerate_integrals(H.Pattern("****", 2), 4)

    def partial(sp, shard, n_shards):
        full = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], step, sp, dielectric=10.89))
        return np.where(density_shard_of_steps(sp, 4, n_shards) == shard, full, 0)

    full = multi.compute_density_sharded(partial, specs)
    if rank == 0:
        np.save(result_path, full)
    dist.barrier()
    dist.destroy_process_group()


def test_density_split_allreduce_matches_single_process(tmp_path):
    from coulombo_lattice_b200 import synth
    from oracle import host as H
    port = _free_port()
    out = str(tmp_path / "full.npy")
    mp.start_processes(_density_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    d = synth.build("c1", cells=(2, 2, 2))
    specs = H.enumerate_integrals(H.Pattern("****", 2), 4)
    want = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], (synth.A_ZB / 4,) * 3,
                                        specs, dielectric=10.89))
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_density_shards_cover_every_integral_once():
    from oracle import host as H
    specs = H.enumerate_integrals(H.Pattern("eeee,hhhh,ehhe,eheh", 4), 8)
    for world in (1, 2, 3, 8, 50):
        sh = density_shard_of_steps(specs, 8, world)
        assert sh.min() >= 0 and sh.max() < world


def test_round_masks_cover_every_round_once():
    for world in range(1, 9):
        masks = [multi.round_mask(r, world) for r in range(world)]
        assert sum(masks) == 0xFF
        for a in range(world):
            for b in range(a + 1, world):
                assert masks[a] & masks[b] == 0


def test_partition_structures():
    costs = [48 ** 3 * 36, 160 ** 3 * 36, 64 ** 3 * 36, 96 ** 3 * 36, 120 ** 3 * 36, 80 ** 3 * 36]
    parts = multi.partition_structures(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= 1.5 * sum(costs) / 3 + max(costs)


def test_round_split_allreduce_matches_single_process(tmp_path):
    from coulombo_lattice_b200 import synth
    from oracle import host as H
    port = _free_port()
    out = str(tmp_path / "full.npy")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    d = synth.build("c1", cells=(2, 2, 2))
    specs = H.enumerate_integrals(H.Pattern("****", 2), 4)
    want = np.array(H.compute_integrals(list(d["states"]), d["cells_idx"], d["dims"], (synth.A_ZB / 4,) * 3,
                                        specs, dielectric=10.89))
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
