"""Worlds sharded over ranks (the multi-GPU layout of the many-worlds
workload), on the CPU: two `gloo` ranks each take their block of worlds,
step it with the dynamics stage of the C restatement, and gather the
per-world results; rank 0 checks them against one process stepping every
world, and against the reference's own captured outputs."""
import os
import pickle
import socket

import numpy as np
import pytest

import dynio
import reflib
from reactphysics3d_b200 import dynamics as D
from reactphysics3d_b200 import shard

GOLDEN = reflib.ROOT + "/tests/golden/np_dynamics.npz"


def test_blocks_cover_every_world_once():
    rng = np.random.default_rng(3)
    for n in (0, 1, 2, 3, 7, 64, 4096):
        costs = rng.integers(20, 201, n)
        for w in (1, 2, 3, 4, 8):
            b = shard.block_bounds(costs, w)
            assert len(b) == w + 1 and b[0] == 0 and b[-1] == n
            assert all(b[k] <= b[k + 1] for k in range(w)), (n, w, b)
            if n >= w:
                assert all(b[k] < b[k + 1] for k in range(w)), (n, w, b)
            got = np.concatenate([np.arange(*shard.rank_block(costs, r, w)) for r in range(w)]) if n else []
            assert np.array_equal(got, np.arange(n))


def test_blocks_are_balanced_by_cost():
    costs = np.random.default_rng(5).integers(20, 201, 4096)
    for w in (2, 4, 8):
        b = shard.block_bounds(costs, w)
        sums = [costs[b[r]:b[r + 1]].sum() for r in range(w)]
        # a contiguous split is off by at most one world's cost per boundary
        assert max(sums) - min(sums) <= 2 * costs.max(), sums


def test_bad_arguments():
    with pytest.raises(ValueError):
        shard.block_bounds([1, 2], 0)
    with pytest.raises(ValueError):
        shard.rank_block([1, 2], 2, 2)
    with pytest.raises(ValueError):
        shard.block_bounds([1, -1], 2)


def _worlds():
    z = np.load(GOLDEN)
    caps = [dynio.capture(z, n) for n in dynio.cases(z)]
    # 11 worlds of uneven sizes (the captures repeated), so blocks differ in count
    order = [0, 3, 1, 4, 2, 2, 0, 4, 1, 3, 4]
    return [caps[k] for k in order]


def _step(caps):
    import reflib as R
    from reactphysics3d_b200 import dynamics as DD
    port = R.PortEngine()
    worlds = [DD.world_from_capture(c) for c in caps]
    batch, layout = DD.batch_worlds(worlds)
    dynio.run_oracle(port.lib, DD.params_from_capture(caps[0]), batch)
    return [{k: np.asarray(v).copy() for k, v in w.a.items()} for w in DD.unbatch_worlds(batch, layout)]


def _rank_main(rank, world_size, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        caps = _worlds()
        costs = [len(c["in_body_mass"]) for c in caps]
        lo, hi = shard.rank_block(costs, rank, world_size)
        mine = _step(caps[lo:hi])
        everyone = shard.gather_objects((lo, hi, mine))
        slowest = shard.max_over_ranks(float(rank + 1))
        if rank == 0:
            with open(out_path, "wb") as fh:
                pickle.dump((everyone, slowest), fh)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_match_one_process(tmp_path, port):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.pkl")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    with open(out, "rb") as fh:
        everyone, slowest = pickle.load(fh)
    assert slowest == 2.0
    caps = _worlds()
    assert [b[:2] for b in everyone] == [(0, everyone[0][1]), (everyone[0][1], len(caps))]
    assert 0 < everyone[0][1] < len(caps)
    gathered = [w for _, _, ws in everyone for w in ws]
    single = _step(caps)
    assert len(gathered) == len(single) == len(caps)
    for g, s, cap in zip(gathered, single, caps):
        # the stage's outputs (index fields such as the collider -> body row
        # keep the numbering of the batch they were stepped in)
        for k in list(dynio.OUT_CHECKS) + ["inv_inertia_world"]:
            assert np.array_equal(np.asarray(g[k]).view(np.uint8), np.asarray(s[k]).view(np.uint8)), k
        w = D.DynWorld(g, int(cap["in_body_nb_enabled"][0]), int(cap["in_collider_nb_enabled"][0]))
        assert dynio.mismatches(w, cap) == {}
